"""Map-chunked FP64 CBPDN iterations in torch on the CPU (multi-threaded).

TEST INFRASTRUCTURE ONLY.  Like ``cbpdn_oracle`` this is the checker: only
the test suite and the CPU legs of ``bench.py`` import it; the product never
does.

``cbpdn_oracle.admm_lean`` restated with torch float64 CPU tensors, whose
element-wise operations and FFTs use every host thread: the same iterations
(sporco_cuda/src/cbpdn.cu:319-567, cbpdn_grd.cu:358-606), the same
stopping test and adaptive rho (the shared ``cbpdn_oracle._finalize``), the
same y-step (``cbpdn_oracle.y_step`` restated), maps processed in chunks so
that only Y and U are full-size arrays.  The CPU baseline of the benchmark
times it, and the benchmark's relative error compares the GPU result with
it on the benchmark's own problem sizes (2048 x 2048 with 256 maps needs
about 20 GB of host memory here, against more than 80 GB for ``admm``).
``tests/test_oracle_kat.py`` holds it to ``cbpdn_oracle.admm``.
"""

from __future__ import annotations

import numpy as np
import torch

from . import cbpdn_oracle as O

F64 = torch.float64


def _pad_spectrum(D, H, W):
    """rfft2 of filters (m, Kr, Kc) zero-padded to (H, W) (cuda_Pad_Dict +
    R2C, cbpdn_kernels.cu:602-615, cbpdn.cu:277-289)."""
    m, Kr, Kc = D.shape
    P = torch.zeros((m, H, W), dtype=F64)
    P[:, :Kr, :Kc] = D
    return torch.fft.rfft2(P)


def _available_bytes():
    try:
        import psutil
        return int(psutil.virtual_memory().available)
    except Exception:  # pragma: no cover
        return 0


def admm_lean(prob: O.Problem, res: O.Resolved, xi: float, chunk=16, record=True, keep=None):
    """The iterations of ``cbpdn_oracle.admm_lean`` in torch (see there).

    keep: hold the dictionary spectra and pass 1's b for pass 2 instead of
    recomputing them (two full-size complex arrays more); None: when they
    fit in half of the host memory that is available."""
    it = iterate(prob, res, xi, chunk=chunk, record=record, keep=keep)
    for state in it:
        pass
    return state["Y"].numpy(), {"iterations": state["k"], "rho": state["rho"],
                                "hist": state["hist"]}


def iterate(prob: O.Problem, res: O.Resolved, xi: float, chunk=16, record=True, keep=None):
    """Generator of the iterations of :func:`admm_lean`: yields the state
    (k, rho, Y, U, hist) after every iteration, until the stopping test or
    MaxMainIter ends the solve."""
    D = torch.as_tensor(np.ascontiguousarray(prob.D), dtype=F64)
    S = torch.as_tensor(np.ascontiguousarray(prob.S), dtype=F64)
    M = D.shape[0]
    H, W = S.shape
    n = M * H * W
    Sf = torch.fft.rfft2(S)
    grd = prob.wgrd is not None
    Gh = torch.as_tensor(O.gradient_spectrum(H, W), dtype=F64)[None] if grd else None
    wgrd = torch.as_tensor(np.asarray(prob.wgrd, dtype=np.float64)) if grd else None
    wl1 = torch.as_tensor(np.asarray(prob.wl1, dtype=np.float64))
    mask = torch.as_tensor(prob.mask, dtype=F64) if prob.mask is not None else None
    alpha = res.RelaxParam
    rho = res.rho0
    Y = torch.zeros((M, H, W), dtype=F64)
    U = torch.zeros((M, H, W), dtype=F64)
    hist = {"r": [], "s": [], "rho": [], "epri": [], "edua": []}
    chunks = [(m0, min(M, m0 + chunk)) for m0 in range(0, M, chunk)]
    spec_bytes = M * H * (W // 2 + 1) * 16
    if keep is None:
        keep = 2 * spec_bytes + 2 * M * H * W * 8 < 0.5 * _available_bytes()
    Dfull = _pad_spectrum(D, H, W) if keep else None
    bkeep = torch.empty((M, H, W // 2 + 1), dtype=torch.complex128) if keep else None

    def dict_chunk(m0, m1):
        return Dfull[m0:m1] if keep else _pad_spectrum(D[m0:m1], H, W)

    def d_chunk(m0, m1):
        if not grd:
            return rho
        return prob.mu * wgrd[m0:m1].reshape(-1, 1, 1) * Gh + rho

    def y_step(V, m0, m1):
        w = wl1[m0:m1] if wl1.shape[0] > 1 else wl1
        Yn = torch.sign(V) * torch.clamp(torch.abs(V) - (prob.lmbda / rho) * w, min=0.0)
        if prob.nonneg:
            Yn.clamp_(min=0.0)
        if prob.nobndry is not None:
            Kr, Kc = prob.nobndry
            if Kr > 1:
                Yn[:, H - (Kr - 1):, :] = 0.0
            if Kc > 1:
                Yn[:, :, W - (Kc - 1):] = 0.0
        if mask is not None and m0 == 0:
            Yn[0] = (1.0 - mask) * V[0]
        return Yn

    k = 0
    for k in range(1, res.MaxMainIter + 1):
        num = torch.zeros((H, W // 2 + 1), dtype=torch.complex128)
        sden = torch.zeros((H, W // 2 + 1), dtype=F64)
        for m0, m1 in chunks:
            Dc = dict_chunk(m0, m1)
            d = d_chunk(m0, m1)
            b = torch.conj(Dc) * Sf[None] + rho * torch.fft.rfft2(Y[m0:m1] - U[m0:m1])
            if keep:
                bkeep[m0:m1] = b
            num += torch.sum(Dc * b / d, dim=0)
            sden += torch.sum((Dc.real ** 2 + Dc.imag ** 2) / d, dim=0)
        cb = num / (1.0 + sden)
        sums = [0.0] * 5
        for m0, m1 in chunks:
            Dc = dict_chunk(m0, m1)
            d = d_chunk(m0, m1)
            if keep:
                b = bkeep[m0:m1]
            else:
                b = torch.conj(Dc) * Sf[None] + rho * torch.fft.rfft2(Y[m0:m1] - U[m0:m1])
            X = torch.fft.irfft2((b - torch.conj(Dc) * cb[None]) / d, s=(H, W))
            Yc, Uc = Y[m0:m1], U[m0:m1]
            V = (alpha * X + (1.0 - alpha) * Yc if alpha != 1.0 else X) + Uc
            Yn = y_step(V, m0, m1)
            Un = V - Yn
            sums[0] += float(torch.sum(X * X))
            sums[1] += float(torch.sum(Yn * Yn))
            sums[2] += float(torch.sum(Un * Un))
            sums[3] += float(torch.sum((X - Yn) ** 2))
            sums[4] += float(torch.sum((Yc - Yn) ** 2))
            Y[m0:m1] = Yn
            U[m0:m1] = Un
        rho, rsf, stop = O._finalize(sums, rho, k, n, res, xi, hist if record else None)
        if rsf != 1.0:
            U /= rsf
        yield {"k": k, "rho": rho, "Y": Y, "U": U, "hist": hist}
        if stop:
            break


def problem(variant, D, S, lmbda, opt, mu=0.0, W=None):
    """(Problem, Resolved options, xi) of the oracle entry point `variant`
    (cbpdn, cbpdngrd, cbpdnmsk, cbpdngrdmsk; D (Kr, Kc, M), S (H, W), mask W
    for the masked ones), as ``cbpdn_oracle`` builds them."""
    grd = variant in ("cbpdngrd", "cbpdngrdmsk")
    ams = variant in ("cbpdnmsk", "cbpdngrdmsk")
    Dk = np.asarray(D, dtype=np.float32)
    wl1 = wg = None
    if ams:
        Dk, wl1, wg = O._ams(Dk, opt, grd)
    M = Dk.shape[2]
    res = O.resolve_options(opt, lmbda)
    wl1a = O._l1_weight({"L1Weight": wl1} if wl1 is not None else opt, M)
    wga = O._grad_weight({"GradWeight": wg} if wg is not None else opt, M) if grd else None
    mask = None
    if ams and W is not None and np.asarray(W).size > 1:
        mask = np.ascontiguousarray(W, dtype=np.int32).astype(np.float64)
    prob = O.Problem(D=np.moveaxis(Dk, 2, 0).astype(np.float64),
                     S=np.asarray(S, dtype=np.float32).astype(np.float64),
                     lmbda=float(np.float32(lmbda)), mu=float(np.float32(mu)), wl1=wl1a,
                     wgrd=wga, mask=mask,
                     nonneg=bool(O._get(opt, "NonNegCoef", False)),
                     nobndry=tuple(Dk.shape[0:2]) if O._get(opt, "NoBndryCross", False) else None)
    return prob, res, O.rsdl_target(res, lmbda)


def solve(variant, D, S, lmbda, opt, mu=0.0, W=None, chunk=16, keep=None):
    """The oracle entry point ``variant`` (see :func:`problem`) with these
    iterations; returns (X (H, W, M), info), the AMS map dropped."""
    prob, res, xi = problem(variant, D, S, lmbda, opt, mu=mu, W=W)
    Y, info = admm_lean(prob, res, xi, chunk=chunk, keep=keep)
    X = np.moveaxis(Y, 0, 2)
    return (X[..., 1:] if variant in ("cbpdnmsk", "cbpdngrdmsk") else X), info


def objective(Dm, S, Y, lmbda, mu=0.0, wgrd=None, mask=None, chunk=16):
    """``cbpdn_oracle.objective`` computed chunk by chunk over the maps, in
    torch float64 on the CPU: Dm (M, Kr, Kc), S (H, W), Y (M, H, W) (any
    float dtype; converted per chunk)."""
    M = Dm.shape[0]
    H, W = S.shape
    D = torch.as_tensor(np.ascontiguousarray(Dm), dtype=F64)
    acc = torch.zeros((H, W // 2 + 1), dtype=torch.complex128)
    l1 = 0.0
    gr = 0.0
    for m0 in range(0, M, chunk):
        m1 = min(M, m0 + chunk)
        Yc = torch.as_tensor(np.ascontiguousarray(Y[m0:m1])).to(F64)
        acc += torch.sum(_pad_spectrum(D[m0:m1], H, W) * torch.fft.rfft2(Yc), dim=0)
        l1 += float(torch.sum(torch.abs(Yc)))
        if wgrd is not None and mu != 0.0:
            g = torch.as_tensor(np.asarray(wgrd, dtype=np.float64)[m0:m1]).reshape(-1, 1, 1)
            a = Yc - torch.roll(Yc, 1, dims=2)
            b = Yc - torch.roll(Yc, 1, dims=1)
            gr += float(torch.sum(g * (a * a + b * b)))
    e = torch.fft.irfft2(acc, s=(H, W)) - torch.as_tensor(np.asarray(S, dtype=np.float64))
    if mask is not None:
        e = e * torch.as_tensor(np.asarray(mask, dtype=np.float64))
    return 0.5 * float(torch.sum(e * e)) + float(lmbda) * l1 + 0.5 * float(mu) * gr
