"""Parity of the kernel instantiations the benchmark runs, at the benchmark's
image sizes, against the FP64 oracle (iteration counts cut so that the
oracle finishes in seconds).

* 512 x 512, 100 filters 12 x 12 (the gradient-regularised and masked
  solves of the 512 x 512 benchmark): ``col_kernel<COL_SOLVE_G16, 512>``,
  ``col_kernel<COL_SOLVE_C16, 512>``, ``row_kernel<ROW_ITER, 512>`` and the
  rho fix-up ``row_kernel<ROW_FIXUP, 512>``;
* 2048 x 2048 and 1024 x 1024 with 16 x 16 filters (the kernels of the
  2048 x 2048, 256-filter benchmark at fewer filters):
  ``col_kernel<COL_SOLVE_C16, 2048|1024>``, the radix-16 row pass with the
  register hand-over ``row_kernel<ROW_ITER, 2048|1024>`` and the fix-up from
  the state ``row_kernel<ROW_FIXUP, 2048|1024>``.

Every case runs with adaptive rho, and checks that rho changed (so the
fix-up ran), that the rho trajectory follows the oracle's, the relative
error of the coefficient maps (<= 1e-4) and of the functional (<= 1e-6).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import sporco_cuda.cbpdn as cb
from oracle import cbpdn_oracle as O

REL_TOL = 1e-4
FUNC_TOL = 1e-6


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def _synth(H, W, M, K, density, seed):
    """The benchmark's synthetic problem: unit-norm Gaussian filters,
    Bernoulli x Gaussian maps, S = sum_m d_m * x_m + N(0, 0.01^2), mean
    removed (float64 FFTs, float32 result)."""
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((K, K, M))
    D /= np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))
    Sf = np.zeros((H, W // 2 + 1), np.complex128)
    for m0 in range(0, M, 16):
        m1 = min(M, m0 + 16)
        X0 = (rng.random((m1 - m0, H, W)) < density) * rng.standard_normal((m1 - m0, H, W))
        Df = np.fft.rfft2(np.moveaxis(D[..., m0:m1], 2, 0), s=(H, W))
        Sf += np.sum(Df * np.fft.rfft2(X0), axis=0)
    s = np.fft.irfft2(Sf, s=(H, W)) + 0.01 * rng.standard_normal((H, W))
    return D.astype(np.float32), (s - s.mean()).astype(np.float32)


def _device_solve(D, S, lam, opt, mu=0.0, grd=False, mask=None):
    """The torch path with per-iteration statistics: (X (H, W, M), rho per
    iteration)."""
    Dm = torch.tensor(np.moveaxis(D, 2, 0).copy(), device="cuda")
    St = torch.tensor(S, device="cuda")[None]
    l1 = 1.0
    if mask is not None:
        Dm = torch.cat((torch.zeros((1,) + Dm.shape[1:], device="cuda"), Dm), 0)
        Dm[0, 0, 0] = 1.0
        l1 = np.ones(Dm.shape[0], np.float32)
        l1[0] = 0.0
        mask = torch.tensor(mask, device="cuda").to(torch.int32)[None]
    ds = cb.prepare_device(Dm, St, lam, opt, mu=mu, grd=grd, l1=l1, mask=mask,
                           record_itstat=True)
    Y = ds.run()[0]
    st = ds.state()
    k = st["iterations"][0]
    X = Y.permute(1, 2, 0).cpu().numpy()
    if mask is not None:
        X = X[..., 1:]
    return X, st["itstat"][0, :k, 2]


def _check(D, S, X, Xo, rho, info, lam, mu=0.0, grd=False, mask=None):
    rho_o = np.asarray(info["hist"]["rho"])
    assert len(rho) == len(rho_o)
    assert np.unique(rho_o).size > 1, "rho never changed: the fix-up did not run"
    # rho is a product of continuous AutoScaling factors sqrt(r / (s xi)),
    # and the dual residual s is the norm of the change of Y between two
    # iterations: late in a solve it is small and carries the float32 error
    # of both iterates, which grows along the trajectory (up to 1.4e-4 here
    # at 25 iterations); 5e-4 still separates that from a flipped decision,
    # which differs by a factor of about 1.2 or more
    np.testing.assert_allclose(rho, rho_o, rtol=5e-4)
    assert _rel(X, Xo) < REL_TOL
    Dm = np.moveaxis(D, 2, 0).astype(np.float64)
    Sd = S.astype(np.float64) * (mask if mask is not None else 1.0)
    kw = dict(mu=mu, wgrd=np.ones(D.shape[2]) if grd else None, mask=mask)
    J = O.objective(Dm, Sd, np.moveaxis(X.astype(np.float64), 2, 0), np.float32(lam), **kw)
    Jo = O.objective(Dm, Sd, np.moveaxis(np.asarray(Xo, np.float64), 2, 0), np.float32(lam), **kw)
    assert abs(J - Jo) / Jo < FUNC_TOL, (J, Jo)


@pytest.fixture(scope="module")
def problem_512():
    return _synth(512, 512, 100, 12, 0.005, 12346)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["cbpdngrd", "cbpdnmsk"])
def test_512x512_m100_autorho(problem_512, variant):
    """The 512 x 512, M = 100 benchmark solves (lambda 0.05, mu 0.1, mask
    Bernoulli(0.7)) cut to 25 iterations."""
    D, S = problem_512
    lam, mu = 0.05, 0.1
    opt = {"MaxMainIter": 25, "RelStopTol": 0.0, "RelaxParam": 1.8, "rho": None,
           "AutoRho": {"Enabled": True, "Period": 1, "Scaling": 1000.0, "RsdlRatio": 1.2,
                       "AutoScaling": True}}
    if variant == "cbpdngrd":
        X, rho = _device_solve(D, S, lam, opt, mu=mu, grd=True)
        Xo, info = O.cbpdngrd(D, S, lam, mu, opt, return_info=True)
        _check(D, S, X, Xo, rho, info, lam, mu=mu, grd=True)
        Xn = cb.cbpdngrd(D, S, lam, mu, opt)  # the reference-facing C ABI
    else:
        Wm = (np.random.default_rng(3).random(S.shape) < 0.7).astype(np.float32)
        X, rho = _device_solve(D, S * Wm, lam, opt, mask=Wm)
        Xo, info = O.cbpdnmsk(D, S * Wm, Wm, lam, opt, return_info=True)
        _check(D, S, X, Xo, rho, info, lam, mask=Wm)
        Xn = cb.cbpdnmsk(D, S * Wm, Wm, lam, opt)
    assert _rel(Xn, Xo) < REL_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("size,M,variant", [(2048, 12, "cbpdn"), (1024, 16, "cbpdn"),
                                            (1024, 16, "cbpdnmsk")])
def test_radix16_row_plans_and_convolution_solve(size, M, variant):
    """16 x 16 filters at the 2048 x 2048 benchmark's lambda, adaptive rho,
    10 iterations."""
    D, S = _synth(size, size, M, 16, 0.01, 12349 + size)
    lam = 0.02
    opt = {"MaxMainIter": 10, "RelStopTol": 0.0, "RelaxParam": 1.8, "rho": None,
           "AutoRho": {"Enabled": True, "Period": 1, "Scaling": 1000.0, "RsdlRatio": 1.2,
                       "AutoScaling": True}}
    if variant == "cbpdn":
        X, rho = _device_solve(D, S, lam, opt)
        Xo, info = O.cbpdn(D, S, lam, opt, return_info=True)
        _check(D, S, X, Xo, rho, info, lam)
    else:
        Wm = (np.random.default_rng(5).random(S.shape) < 0.7).astype(np.float32)
        X, rho = _device_solve(D, S * Wm, lam, opt, mask=Wm)
        Xo, info = O.cbpdnmsk(D, S * Wm, Wm, lam, opt, return_info=True)
        _check(D, S, X, Xo, rho, info, lam, mask=Wm)
