"""Known-answer tests that pin the oracle independently of the reference."""

import numpy as np
import pytest

from oracle import cbpdn_oracle as O


def _impulse(K=5):
    D = np.zeros((K, K, 1), np.float32)
    D[0, 0, 0] = 1.0
    return D


def test_impulse_dictionary_gives_soft_threshold():
    rng = np.random.default_rng(1)
    S = rng.standard_normal((24, 19)).astype(np.float32)
    lam = 0.4
    X = O.cbpdn(_impulse(), S, lam, {"MaxMainIter": 400, "RelStopTol": 1e-9,
                                     "AutoRho": {"Enabled": True}})
    ref = np.sign(S) * np.maximum(np.abs(S) - np.float32(lam), 0)
    np.testing.assert_allclose(X[..., 0], ref, atol=1e-6)


def test_gradreg_impulse_closed_form():
    """delta dictionary, lambda = 0: X^ = S^ / (1 + mu |G|^2)."""
    rng = np.random.default_rng(2)
    H, W = 16, 21
    S = rng.standard_normal((H, W)).astype(np.float32)
    mu = 0.7
    X = O.cbpdngrd(_impulse(3), S, 0.0, mu, {"MaxMainIter": 300, "RelStopTol": 1e-12,
                                               "rho": 1.0, "AutoRho": {"Enabled": False}})
    Gh = O.gradient_spectrum(H, W)
    ref = np.fft.irfft2(np.fft.rfft2(S.astype(np.float64)) / (1 + np.float32(mu) * Gh), s=(H, W))
    np.testing.assert_allclose(X[..., 0], ref, atol=1e-6)


def test_sherman_morrison_matches_dense_solve():
    rng = np.random.default_rng(3)
    M = 6
    for grd in (False, True):
        Df = rng.standard_normal(M) + 1j * rng.standard_normal(M)
        b = rng.standard_normal(M) + 1j * rng.standard_normal(M)
        rho = 1.7
        d = rho + (0.3 * rng.random(M) if grd else 0.0)
        A = np.outer(np.conj(Df), Df) + np.diag(d * np.ones(M))
        x_dense = np.linalg.solve(A, b)
        cb = np.sum(Df * b / d) / (1 + np.sum(np.abs(Df) ** 2 / d))
        x_sm = (b - np.conj(Df) * cb) / d
        np.testing.assert_allclose(x_sm, x_dense, rtol=1e-12, atol=1e-12)


def test_kkt_at_convergence():
    """D^T (D x - s) + lambda w sign(x) = 0 on the support, |.| <= lambda off it."""
    rng = np.random.default_rng(4)
    H, W, M, K = 20, 20, 3, 4
    D = rng.standard_normal((K, K, M)).astype(np.float32)
    S = rng.standard_normal((H, W)).astype(np.float32)
    lam = 0.5
    X = O.cbpdn(D, S, lam, {"MaxMainIter": 3000, "RelStopTol": 1e-10, "rho": 5.0,
                            "AutoRho": {"Enabled": False}})
    Xm = np.moveaxis(X, 2, 0)
    Df = O.pad_dict_spectrum(np.moveaxis(D, 2, 0).astype(np.float64), H, W)
    R = O.irfft2(np.sum(Df * O.rfft2(Xm), axis=0), (H, W)) - S
    G = O.irfft2(np.conj(Df) * O.rfft2(R)[None], (H, W))
    lam32 = float(np.float32(lam))
    on = np.abs(Xm) > 1e-6
    assert np.max(np.abs(G[on] + lam32 * np.sign(Xm[on]))) < 1e-6
    assert np.max(np.abs(G[~on])) < lam32 + 1e-6


def test_mask_all_ones_tends_to_unmasked_objective():
    rng = np.random.default_rng(5)
    H, W, M, K = 16, 16, 3, 3
    D = rng.standard_normal((K, K, M)).astype(np.float32)
    S = rng.standard_normal((H, W)).astype(np.float32)
    opt = {"MaxMainIter": 3000, "RelStopTol": 1e-9, "rho": 3.0, "AutoRho": {"Enabled": False}}
    X1 = O.cbpdn(D, S, 0.2, opt)
    X2 = O.cbpdnmsk(D, S, np.ones((H, W), np.float32), 0.2, opt)
    Dm = np.moveaxis(D, 2, 0).astype(np.float64)
    J1 = O.objective(Dm, S, np.moveaxis(X1, 2, 0), np.float32(0.2))
    J2 = O.objective(Dm, S, np.moveaxis(X2, 2, 0), np.float32(0.2))
    assert abs(J1 - J2) / J1 < 1e-4


def test_objective_parseval_matches_spatial():
    rng = np.random.default_rng(6)
    D = rng.standard_normal((3, 3, 2))
    S = rng.standard_normal((9, 8))
    Y = rng.standard_normal((2, 9, 8))
    J = O.objective(np.moveaxis(D, 2, 0), S, Y, 0.3)
    # direct circular convolution
    rec = np.zeros((9, 8))
    for m in range(2):
        for i in range(3):
            for j in range(3):
                rec += D[i, j, m] * np.roll(np.roll(Y[m], i, axis=0), j, axis=1)
    ref = 0.5 * np.sum((rec - S) ** 2) + 0.3 * np.sum(np.abs(Y))
    assert abs(J - ref) < 1e-9 * abs(ref)


@pytest.mark.parametrize("lam,std,expect", [(0.1, False, 1 + 18.3 ** 0.0), (0.05, True, 1.0)])
def test_rsdl_target(lam, std, expect):
    r = O.resolve_options({"AutoRho": {"StdResiduals": std}}, lam)
    assert abs(O.rsdl_target(r, lam) - expect) < 1e-6 * expect


def test_option_marshalling_rounds_like_the_reference():
    r = O.resolve_options({"RelaxParam": 1.8, "rho": None}, 0.1)
    assert r.RelaxParam == float(np.float32(1.8))
    assert r.rho0 == float(np.float32(50 * float(np.float32(0.1)) + 1))
