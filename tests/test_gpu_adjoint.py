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
# filters at 128 x 128 (16 taps) and at 256 x 256 with 32 filters (the
# differentiable benchmark's filters), the first over 200 iterations (15
# segments of 14).
SHAPES = [(2, 24, 20, 3, 5, 12), (1, 32, 30, 4, 5, 10), (2, 64, 64, 8, 7, 9),
          (1, 128, 128, 8, 11, 200), (1, 256, 256, 32, 11, 10)]


def _gpu_masks(D, S, iters):
    """The shrinkage pattern Y_k != 0 of the GPU's own forward iterations,
    k = 1..iters (the unrolled forward is deterministic, so the first k
    iterations of every run are the same)."""
    import sporco_cuda.adjoint as adj
    Dt, St = torch.tensor(D, device="cuda"), torch.tensor(S, device="cuda")
    masks = []
    for k in range(1, iters + 1):
        X = adj.cbpdn_unrolled(Dt, St, LAM, dict(_opt(), MaxMainIter=k))
        masks.append((X != 0).permute(0, 3, 1, 2).cpu())
    return masks


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["default", "transform", "traced"])
@pytest.mark.parametrize("shape", SHAPES)
def test_unrolled_gradients_match_fp64_autograd_and_fd(shape, form, monkeypatch):
    """The hand-written adjoint against torch FP64 autograd and FP64 central
    differences.

    A float32 forward and a float64 forward of the same iterations can put
    an element on different sides of its shrinkage threshold when it lies
    within rounding of it; the unrolled loss has a kink there and the two
    gradients then differ by far more than rounding (1e-3 on the larger
    shapes).  The reference is therefore the FP64 loss taken along the GPU
    forward's own shrinkage pattern (identical to the plain FP64 loss
    wherever the patterns agree, smooth in D and S around the point), and
    the plain FP64 gradient is compared as well whenever the FP64 forward
    produces the same pattern (the L1 term likewise takes the GPU's signs of
    Y_K, the value of |Y_K| wherever the signs agree, so that an active
    coefficient next to zero puts no kink inside the difference step).
    "transform" forces the transform-solve
    adjoint (SPORCO_B200_ADJOINT) where the convolution form would run;
    "traced" keeps every step's trace in the forward pass (one segment) so
    that the backward pass recomputes nothing."""
    import sporco_cuda.adjoint as adj
    B, H, W, M, K, iters = shape
    if shape[0:2] == (2, 24) and form != "default":
        pytest.skip("the transform form is the only one here")
    if form == "transform":
        monkeypatch.setenv("SPORCO_B200_ADJOINT", "transform")
    ckpt = "all" if form == "traced" else "sqrt"
    D, S, Sc = _problem(B, H, W, M, K)
    lam, rho, alpha = _consts()
    opt = dict(_opt(), MaxMainIter=iters)
    Dg = torch.tensor(D, device="cuda", requires_grad=True)
    Sg = torch.tensor(S, device="cuda", requires_grad=True)
    X = adj.cbpdn_unrolled(Dg, Sg, LAM, opt, checkpoints=ckpt)
    R = adj.reconstruct(Dg, X)
    L = torch.sum((R - torch.tensor(Sc, device="cuda")) ** 2) + BETA * torch.sum(torch.abs(X))
    L.backward()
    masks = _gpu_masks(D, S, iters)
    Sc64 = torch.tensor(Sc, dtype=torch.float64)
    sgn = torch.sign(X.detach()).permute(0, 3, 1, 2).double().cpu()  # the GPU's Y_K signs

    def ref_grads(use_masks):
        Dt = torch.tensor(D, dtype=torch.float64, requires_grad=True)
        St = torch.tensor(S, dtype=torch.float64, requires_grad=True)
        Lr = A.loss(Dt, St, Sc64, lam, rho, alpha, iters, BETA,
                    masks=masks if use_masks else None, l1sign=sgn if use_masks else None)
        Lr.backward()
        return float(Lr), Dt.grad, St.grad

    Lm, gDm, gSm = ref_grads(True)
    assert abs(float(L.detach()) - Lm) / Lm < 1e-5
    for g, r in ((Dg.grad, gDm), (Sg.grad, gSm)):
        g = g.double().cpu()
        rel = float(torch.linalg.norm(g - r) / torch.linalg.norm(r))
        assert rel < 1e-4, rel
    # the plain FP64 unrolled solve, where its shrinkage pattern is the GPU's
    trace = []
    A.unrolled(torch.tensor(D, dtype=torch.float64), torch.tensor(S, dtype=torch.float64), lam,
               rho, alpha, iters, trace=trace)
    if all(torch.equal(y != 0, m) for y, m in zip(trace, masks)):
        Lp, gDp, gSp = ref_grads(False)
        for g, r in ((Dg.grad, gDp), (Sg.grad, gSp)):
            g = g.double().cpu()
            assert float(torch.linalg.norm(g - r) / torch.linalg.norm(r)) < 1e-4
    # directional central differences of the FP64 loss along the GPU's
    # pattern (and the GPU's signs of Y_K in its L1 term: smooth around the
    # point), against the GPU gradient
    rng = np.random.default_rng(7)
    for g, base, which in ((Dg.grad, D, "D"), (Sg.grad, S, "S")):
        dd = torch.tensor(rng.standard_normal(base.shape))

        def f(x):
            d = torch.tensor(D, dtype=torch.float64) if which == "S" else x
            s = torch.tensor(S, dtype=torch.float64) if which == "D" else x
            return float(A.loss(d, s, Sc64, lam, rho, alpha, iters, BETA, masks=masks,
                                l1sign=sgn))
        x0 = torch.tensor(base, dtype=torch.float64)
        eps = 1e-6
        fp, fm = f(x0 + eps * dd), f(x0 - eps * dd)
        fd = (fp - fm) / (2 * eps)
        gn = g.double().cpu().numpy()
        an = float(np.sum(gn * dd.numpy()))
        # a random direction's derivative can be much smaller than |g| |dd|;
        # the bound is relative to the derivative or to |g| |dd| / sqrt(n),
        # the size of a typical one, whichever is larger
        scale = max(abs(fd), np.linalg.norm(gn) * float(torch.linalg.norm(dd)) /
                    np.sqrt(gn.size))
        assert abs(fd - an) <= 1e-4 * scale, (which, fd, an, scale)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(1, 64, 64, 8, 7, 9), (2, 128, 128, 8, 11, 24)])
def test_checkpoint_spacings_give_identical_results(shape):
    """The backward pass recomputes each segment from its checkpoint (the
    state V) with the trace-keeping twins of the forward's kernels, or,
    with one segment, reads the traces the forward kept: every spacing must
    reproduce the forward's iterates bit for bit, so the output and both
    gradients are identical for every spacing."""
    import sporco_cuda.adjoint as adj
    B, H, W, M, K, iters = shape
    D, S, Sc = _problem(B, H, W, M, K)
    opt = dict(_opt(), MaxMainIter=iters)
    out = {}
    for ckpt in ("sqrt", "all", 2, iters - 1):
        Dg = torch.tensor(D, device="cuda", requires_grad=True)
        Sg = torch.tensor(S, device="cuda", requires_grad=True)
        X = adj.cbpdn_unrolled(Dg, Sg, LAM, opt, checkpoints=ckpt)
        R = adj.reconstruct(Dg, X)
        L = torch.sum((R - torch.tensor(Sc, device="cuda")) ** 2) + BETA * torch.sum(torch.abs(X))
        L.backward()
        out[ckpt] = (X.detach().cpu(), Dg.grad.cpu(), Sg.grad.cpu())
    X0, gD0, gS0 = out["sqrt"]
    for ckpt, (X, gD, gS) in out.items():
        assert torch.equal(X, X0), ckpt
        assert torch.equal(gD, gD0), ckpt
        assert torch.equal(gS, gS0), ckpt
