"""Differentiable CBPDN: the unrolled ADMM solve as a torch.autograd.Function.

No counterpart in the reference.  ``cbpdn_unrolled(D, S, lmbda, opt)`` runs a
fixed number of plain-cbpdn ADMM iterations (``opt['MaxMainIter']``, fixed
rho: adaptive rho and early stopping are not differentiated) and returns the
coefficient maps; its backward pass returns dLoss/dD and dLoss/dS through all
iterations.  The backward pass is hand-written (``csrc/sc_adjoint.cu``): the
shrinkage subgradient mask, the transposed Sherman-Morrison solve (the
system is Hermitian, so it is the forward solve again), the dictionary and
signal gradients accumulated in the frequency domain, and FFTs by this
package's own kernels.  Memory: (Y, U) checkpoints every ceil(sqrt(K))
iterations; each segment is recomputed forward once during the backward pass
and its steps kept while they are reversed.

Shapes: D (Kr, Kc, M), S (B, H, W) or (H, W) float32 CUDA tensors; the result
is (B, H, W, M) (or (H, W, M)).
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from .cbpdn import F32, _opt_get, prepare_device, resolve_options

__all__ = ["cbpdn_unrolled", "reconstruct", "rfft2", "irfft2"]


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def rfft2(x):
    """numpy-convention rfft2 over the last two axes (this package's FFT)."""
    x = x.contiguous().float()
    H, W = x.shape[-2:]
    cnt = x.numel() // (H * W)
    out = torch.empty(x.shape[:-2] + (H, W // 2 + 1), dtype=torch.complex64, device=x.device)
    _lib.check(_lib.sc_rfft2(C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), cnt, H, W,
                             _stream()))
    return out


def irfft2(xf, H, W):
    """numpy-convention irfft2 (normalised by 1/(H W)) back to (.., H, W)."""
    xf = xf.contiguous()
    cnt = xf.numel() // (H * (W // 2 + 1))
    out = torch.empty(xf.shape[:-2] + (H, W), dtype=torch.float32, device=xf.device)
    _lib.check(_lib.sc_irfft2(C.c_void_p(xf.data_ptr()), C.c_void_p(out.data_ptr()), cnt, H, W,
                              _stream()))
    return out


def _dict_spectrum(Dm, H, W):
    """rfft2 of the filters (M, Kr, Kc) zero-padded to (H, W)."""
    M, Kr, Kc = Dm.shape
    P = torch.zeros((M, H, W), dtype=torch.float32, device=Dm.device)
    P[:, :Kr, :Kc] = Dm
    return rfft2(P)


class _Ctx:
    """Per-call constants of the unrolled solve."""

    def __init__(self, Dm, S, lmbda, opt):
        self.B, self.H, self.W = S.shape
        self.M = Dm.shape[0]
        self.Kr, self.Kc = Dm.shape[1:]
        r = resolve_options(opt, float(np.asarray(lmbda).ravel()[0]))
        self.K = int(r["MaxMainIter"])
        self.alpha = float(r["RelaxParam"])
        lam = np.broadcast_to(np.asarray(lmbda, dtype=F32), (self.B,))
        self.lam = torch.as_tensor(lam.copy(), device=S.device)
        rho = _opt_get(opt, "rho")
        self.rho = float(F32(5e1 * float(lam[0]) + 1.0)) if rho is None else float(F32(rho))
        w = _opt_get(opt, "L1Weight")
        self.l1_kind, self.l1_scalar, self.l1w = _lib.SC_L1_SCALAR, float(F32(1.0)), None
        if hasattr(w, "ndim") and np.asarray(w).size > 1:
            w = np.asarray(w, dtype=F32)
            if w.size == self.M:
                self.l1_kind, self.l1w = _lib.SC_L1_PER_MAP, torch.as_tensor(
                    w.ravel().copy(), device=S.device)
            else:
                self.l1_kind = _lib.SC_L1_FULL
                self.l1w = torch.as_tensor(
                    np.ascontiguousarray(np.broadcast_to(np.moveaxis(w, 2, 0),
                                                         (self.M, self.H, self.W))),
                    device=S.device)
        else:
            self.l1_scalar = float(F32(np.asarray(w).ravel()[0]))
        self.Dh = _dict_spectrum(Dm, self.H, self.W)
        self.Sh = rfft2(S)

    def elem(self, mode, X=None, Y=None, U=None, gY=None, gU=None, out=None):
        p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
        _lib.check(_lib.sc_adj_elem(mode, self.B, self.M, self.H, self.W, self.rho, self.alpha,
                                    p(self.lam), self.l1_kind, self.l1_scalar, p(self.l1w),
                                    p(X), p(Y), p(U), p(gY), p(gU), p(out), _stream()))

    def freq(self, mode, io, Xh=None, gDh=None, gSh=None):
        p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
        _lib.check(_lib.sc_adj_freq(mode, self.B, self.M, self.H, self.W, self.rho,
                                    p(self.Dh), p(self.Sh), p(io), p(Xh), p(gDh), p(gSh),
                                    _stream()))

    def step(self, Y, U, keep=False):
        """One ADMM iteration in place on (Y, U); with keep, return (X, X^)."""
        Z = torch.empty_like(Y)
        self.elem(0, Y=Y, U=U, out=Z)
        Zh = rfft2(Z)
        self.freq(0, Zh)                      # Zh <- X^
        X = irfft2(Zh, self.H, self.W)
        self.elem(1, X=X, Y=Y, U=U)
        return (X, Zh) if keep else None


class _Unrolled(torch.autograd.Function):
    @staticmethod
    def forward(ctx, D, S, lmbda, opt):
        Dm = D.detach().permute(2, 0, 1).contiguous().float()
        Sb = S.detach().float().contiguous()
        c = _Ctx(Dm, Sb, lmbda, opt)
        Y = torch.zeros((c.B, c.M, c.H, c.W), device=S.device)
        U = torch.zeros_like(Y)
        seg = max(1, int(math.ceil(math.sqrt(c.K))))
        ckpt = []
        # the fused solver, run segment by segment from each checkpoint
        fopt = dict(opt)
        fopt.update({"RelStopTol": 0.0, "AbsStopTol": 0.0, "rho": c.rho,
                     "AutoRho": {"Enabled": False}})
        l1 = c.l1w if c.l1w is not None else c.l1_scalar
        ds = prepare_device(Dm, Sb, lmbda, fopt, l1=l1, Y=Y, check_every=0)
        ds.prob.U_out = U.data_ptr()
        for k0 in range(0, c.K, seg):
            ckpt.append((k0, Y.clone(), U.clone()))
            ds.opts.max_iter = min(seg, c.K - k0)
            ds.prob.U0 = U.data_ptr() if k0 > 0 else None
            ds.run()
        ctx.c, ctx.seg, ctx.ckpt = c, seg, ckpt
        ctx.dshape = D.shape
        return Y.permute(0, 2, 3, 1).contiguous()

    @staticmethod
    def backward(ctx, gX):
        c = ctx.c
        gY = gX.detach().permute(0, 3, 1, 2).contiguous().float()
        gU = torch.zeros_like(gY)
        Wf = c.W // 2 + 1
        gDh = torch.zeros((c.B, c.M, c.H, Wf), dtype=torch.complex64, device=gY.device)
        gSh = torch.zeros((c.B, c.H, Wf), dtype=torch.complex64, device=gY.device)
        gXs = torch.empty_like(gY)
        for k0, Yc, Uc in reversed(ctx.ckpt):
            k1 = min(c.K, k0 + ctx.seg)
            Y, U = Yc.clone(), Uc.clone()
            steps = []
            for _ in range(k0, k1):
                Yk, Uk = Y.clone(), U.clone()
                X, Xh = c.step(Y, U, keep=True)
                steps.append((Yk, Uk, X, Xh))
            for Yk, Uk, X, Xh in reversed(steps):
                c.elem(2, X=X, Y=Yk, U=Uk, gY=gY, gU=gU, out=gXs)
                Gh = rfft2(gXs)
                c.freq(1, Gh, Xh=Xh, gDh=gDh, gSh=gSh)   # Gh <- Q^
                Q = irfft2(Gh, c.H, c.W)
                c.elem(3, X=Q, gY=gY, gU=gU)
            del steps
        gS = irfft2(gSh, c.H, c.W)
        gDfull = irfft2(torch.sum(gDh, dim=0), c.H, c.W)
        gD = gDfull[:, :c.Kr, :c.Kc].permute(1, 2, 0).contiguous()
        return gD.reshape(ctx.dshape), gS, None, None


def cbpdn_unrolled(D, S, lmbda, opt):
    """Differentiable fixed-iteration cbpdn (see the module docstring)."""
    single = S.ndim == 2
    Sb = S[None] if single else S
    X = _Unrolled.apply(D, Sb, lmbda, opt)
    return X[0] if single else X


class _Reconstruct(torch.autograd.Function):
    @staticmethod
    def forward(ctx, D, X):
        B, H, W, M = X.shape
        Dm = D.detach().permute(2, 0, 1).contiguous().float()
        Dh = _dict_spectrum(Dm, H, W)
        Xh = rfft2(X.detach().permute(0, 3, 1, 2))
        R = irfft2(torch.sum(Dh[None] * Xh, dim=1), H, W)
        ctx.save_for_backward(Dh, Xh)
        ctx.shape = (B, H, W, M) + tuple(D.shape[:2])
        return R

    @staticmethod
    def backward(ctx, gR):
        Dh, Xh = ctx.saved_tensors
        B, H, W, M, Kr, Kc = ctx.shape
        Gh = rfft2(gR.float())
        gX = irfft2(torch.conj(Dh)[None] * Gh[:, None], H, W).permute(0, 2, 3, 1)
        gD = irfft2(torch.sum(Gh[:, None] * torch.conj(Xh), dim=0), H, W)[:, :Kr, :Kc]
        return gD.permute(1, 2, 0).contiguous(), gX.contiguous()


def reconstruct(D, X):
    """sum_m d_m * x_m (circular), differentiable; X (B, H, W, M) -> (B, H, W)."""
    return _Reconstruct.apply(D, X)
