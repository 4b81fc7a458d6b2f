"""FP64 unrolled cbpdn in torch, differentiated by torch autograd.

TEST INFRASTRUCTURE ONLY (imported by the test suite and bench.py's CPU leg).
It restates the plain cbpdn ADMM iteration of ``cbpdn_oracle.admm`` (the
reference's loop, sporco_cuda/src/cbpdn.cu:319-567) with fixed rho, in
float64 torch operations (torch.fft), so that torch autograd gives reference
gradients of any loss of the K-th iterate with respect to D and S.  The
shrinkage is written sign(v) relu(|v| - t), whose autograd subgradient is
1 for |v| > t and 0 elsewhere.
"""

from __future__ import annotations

import numpy as np
import torch


def unrolled(D, S, lmbda, rho, alpha, K, wl1=1.0, masks=None, trace=None):
    """D (Kr, Kc, M), S (B, H, W) float64 tensors -> Y_K (B, M, H, W).

    masks: optional K boolean tensors (B, M, H, W), the shrinkage pattern
    (Y_k != 0) of another computation of the same iterations; step k then
    keeps V - t sign(V) where masks[k] is set and zero elsewhere, so that the
    loss is the smooth function of D and S that coincides with the unrolled
    solve on the region where that computation's thresholds fall the same
    way (its gradient there is what an adjoint of that computation returns).
    trace: optional list that receives Y_k of every step (detached)."""
    B, H, W = S.shape
    Kr, Kc, M = D.shape
    Dp = torch.zeros((M, H, W), dtype=torch.float64)
    Dp = Dp.index_put((torch.arange(M)[:, None, None], torch.arange(Kr)[None, :, None],
                       torch.arange(Kc)[None, None, :]), D.permute(2, 0, 1))
    Df = torch.fft.rfft2(Dp)
    Sf = torch.fft.rfft2(S)
    den = rho + torch.sum(Df.real ** 2 + Df.imag ** 2, dim=0)
    Y = torch.zeros((B, M, H, W), dtype=torch.float64)
    U = torch.zeros_like(Y)
    wl1 = torch.as_tensor(np.asarray(wl1, dtype=np.float64))
    t = lmbda * wl1 / rho
    for k in range(K):
        b = torch.conj(Df)[None] * Sf[:, None] + rho * torch.fft.rfft2(Y - U)
        c = torch.sum(Df[None] * b, dim=1) / den[None]
        Xf = (b - torch.conj(Df)[None] * c[:, None]) / rho
        X = torch.fft.irfft2(Xf, s=(H, W))
        V = alpha * X + (1.0 - alpha) * Y + U
        if masks is None:
            Yn = torch.sign(V) * torch.relu(torch.abs(V) - t)
        else:
            Yn = torch.where(masks[k], V - t * torch.sign(V), torch.zeros_like(V))
        U = V - Yn
        Y = Yn
        if trace is not None:
            trace.append(Y.detach())
    return Y


def reconstruct(D, Y):
    """sum_m d_m * y_m for Y (B, M, H, W)."""
    B, M, H, W = Y.shape
    Kr, Kc, _ = D.shape
    Dp = torch.zeros((M, H, W), dtype=torch.float64)
    Dp = Dp.index_put((torch.arange(M)[:, None, None], torch.arange(Kr)[None, :, None],
                       torch.arange(Kc)[None, None, :]), D.permute(2, 0, 1))
    return torch.fft.irfft2(torch.sum(torch.fft.rfft2(Dp)[None] * torch.fft.rfft2(Y), dim=1),
                            s=(H, W))


def loss(D, S, Sc, lmbda, rho, alpha, K, beta, masks=None, l1sign=None):
    """||D * Y_K - S_clean||^2 + beta ||Y_K||_1 of the unrolled solve (masks:
    see :func:`unrolled`).  l1sign: optional signs (B, M, H, W) of another
    computation's Y_K; ||Y_K||_1 is then taken as sum(l1sign Y_K), its value
    wherever the signs agree, without the kink of |y| at zero."""
    Y = unrolled(D, S, lmbda, rho, alpha, K, masks=masks)
    R = reconstruct(D, Y)
    l1 = torch.sum(torch.abs(Y)) if l1sign is None else torch.sum(l1sign * Y)
    return torch.sum((R - Sc) ** 2) + beta * l1
