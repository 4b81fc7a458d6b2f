"""Differentiable CBPDN: the unrolled ADMM solve as a torch.autograd.Function.

No counterpart in the reference.  ``cbpdn_unrolled(D, S, lmbda, opt)`` runs a
fixed number of plain-cbpdn ADMM iterations (``opt['MaxMainIter']``, fixed
rho: adaptive rho and early stopping are not differentiated) and returns the
coefficient maps; its backward pass returns dLoss/dD and dLoss/dS through all
iterations.  Both passes are single calls into the native library
(``sc_unrolled_forward`` / ``sc_unrolled_backward``): the forward pass is the
solver's own fused iteration, keeping the state V = Y + U every
ceil(sqrt(K)) iterations (``checkpoints="sqrt"``, the default); the backward
pass recomputes each segment once from its checkpoint with the same row pass
(keeping V, the row spectra of X and sc of every step, so that the
recomputed iterates equal the forward's bit for bit) and reverses it with
fused kernels of the same shape as the
forward ones: the shrinkage subgradient mask, the transposed
Sherman-Morrison solve (the system is Hermitian, so it is the forward solve
again) and the dictionary and signal gradients (for filters of at most 16
rows, in the convolution form: the dictionary gradient as correlations over
the filter rows).  ``checkpoints="all"`` keeps every step's trace in the
forward pass instead (memory about K times one iterate and one spectrum),
and the backward pass recomputes nothing; an integer sets the segment
length.

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


def _l1_weight(opt, M, H, W, device):
    """L1Weight of the option dict as the solver's l1 argument."""
    w = _opt_get(opt, "L1Weight")
    if hasattr(w, "ndim") and np.asarray(w).size > 1:
        w = np.asarray(w, dtype=F32)
        if w.size == M:
            return torch.as_tensor(w.ravel().copy(), device=device)
        return torch.as_tensor(np.ascontiguousarray(
            np.broadcast_to(np.moveaxis(w, 2, 0), (M, H, W))), device=device)
    return float(F32(np.asarray(w if w is not None else 1.0).ravel()[0]))


class _Unrolled(torch.autograd.Function):
    @staticmethod
    def forward(ctx, D, S, lmbda, opt, checkpoints="sqrt"):
        Dm = D.detach().permute(2, 0, 1).contiguous().float()
        Sb = S.detach().float().contiguous()
        B, H, W = Sb.shape
        M = Dm.shape[0]
        lam0 = float(np.asarray(lmbda, dtype=F32).ravel()[0])
        r = resolve_options(opt, lam0)
        K = int(r["MaxMainIter"])
        rho = _opt_get(opt, "rho")
        rho = float(F32(5e1 * lam0 + 1.0)) if rho is None else float(F32(rho))
        fopt = dict(opt)
        fopt.update({"RelStopTol": 0.0, "AbsStopTol": 0.0, "rho": rho,
                     "AutoRho": {"Enabled": False}})
        Y = torch.empty((B, M, H, W), device=S.device)
        ds = prepare_device(Dm, Sb, lmbda, fopt, l1=_l1_weight(opt, M, H, W, S.device), Y=Y,
                            check_every=0, workspace=False)
        if checkpoints == "all":
            seg = K
        elif checkpoints == "sqrt":
            seg = max(1, int(math.ceil(math.sqrt(K))))
        else:
            seg = int(checkpoints)
        nbytes = _lib.sc_unrolled_workspace_size(C.byref(ds.prob), C.byref(ds.opts), seg)
        if nbytes == 0:
            _lib.check_last()
        ws = torch.empty(nbytes, dtype=torch.uint8, device=S.device)
        _lib.check(_lib.sc_unrolled_forward(C.byref(ds.prob), C.byref(ds.opts), seg,
                                            C.c_void_p(ws.data_ptr()), nbytes, _stream()))
        ctx.ds, ctx.ws, ctx.seg = ds, ws, seg
        ctx.dshape = D.shape
        return Y.permute(0, 2, 3, 1).contiguous()

    @staticmethod
    def backward(ctx, gX):
        ds = ctx.ds
        B, M, H, W = ds.prob.B, ds.prob.M, ds.prob.H, ds.prob.W
        gY = gX.detach().permute(0, 3, 1, 2).contiguous().float()
        gD = torch.empty((M, ds.prob.Kr, ds.prob.Kc), device=gY.device)
        gS = torch.empty((B, H, W), device=gY.device)
        _lib.check(_lib.sc_unrolled_backward(
            C.byref(ds.prob), C.byref(ds.opts), ctx.seg, C.c_void_p(ctx.ws.data_ptr()),
            ctx.ws.numel(), C.c_void_p(gY.data_ptr()), C.c_void_p(gD.data_ptr()),
            C.c_void_p(gS.data_ptr()), _stream()))
        return gD.permute(1, 2, 0).contiguous().reshape(ctx.dshape), gS, None, None, None


def cbpdn_unrolled(D, S, lmbda, opt, checkpoints="sqrt"):
    """Differentiable fixed-iteration cbpdn (see the module docstring)."""
    single = S.ndim == 2
    Sb = S[None] if single else S
    X = _Unrolled.apply(D, Sb, lmbda, opt, checkpoints)
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
