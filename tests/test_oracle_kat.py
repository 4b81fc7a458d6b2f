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


@pytest.mark.parametrize("variant", ["cbpdn", "cbpdngrd", "cbpdnmsk", "cbpdngrdmsk"])
def test_lean_iterations_equal_full_iterations(variant):
    """admm_lean (maps in chunks, for problems too large for full-size FP64
    temporaries) takes the same iterates as admm: same AutoRho trajectory,
    results equal to summation-order rounding."""
    rng = np.random.default_rng(8)
    H, W, M, K = 24, 20, 7, 4
    D = rng.standard_normal((K, K, M)).astype(np.float32)
    S = rng.standard_normal((H, W)).astype(np.float32)
    Wm = (rng.random((H, W)) < 0.7).astype(np.float32)
    opt = {"MaxMainIter": 25, "RelStopTol": 0.0, "AutoRho": {"Enabled": True},
           "GradWeight": np.linspace(0.5, 1.5, M).astype(np.float32)}
    args = {"cbpdn": (D, S, 0.1, opt), "cbpdngrd": (D, S, 0.1, 0.3, opt),
            "cbpdnmsk": (D, S * Wm, Wm, 0.1, opt), "cbpdngrdmsk": (D, S * Wm, Wm, 0.1, 0.3, opt)}
    f = getattr(O, variant)
    X, info = f(*args[variant], return_info=True)
    Xl, infol = f(*args[variant], return_info=True, lean_chunk=3)
    assert np.linalg.norm(Xl - X) / np.linalg.norm(X) < 1e-11
    np.testing.assert_allclose(infol["hist"]["rho"], info["hist"]["rho"], rtol=1e-12)


def test_nonneg_impulse_dictionary_gives_positive_soft_threshold():
    """NonNegCoef (sporco's projection onto x >= 0): with an impulse
    dictionary the optimum is max(S - lambda, 0)."""
    rng = np.random.default_rng(9)
    S = rng.standard_normal((20, 17)).astype(np.float32)
    lam = 0.3
    opt = {"MaxMainIter": 400, "RelStopTol": 1e-9, "NonNegCoef": True,
           "AutoRho": {"Enabled": True}}
    X = O.cbpdn(_impulse(), S, lam, opt)
    np.testing.assert_allclose(X[..., 0], np.maximum(S - np.float32(lam), 0), atol=1e-6)
    assert X.min() >= 0.0


def test_no_boundary_crossing_impulse_dictionary():
    """NoBndryCross (sporco's zero band where a Kr x Kc filter would cross the
    bottom or right boundary): with an impulse at (0, 0) of a 3 x 4 filter the
    optimum is the soft threshold inside and zero on the last 2 rows and 3
    columns."""
    rng = np.random.default_rng(10)
    H, W = 18, 15
    S = rng.standard_normal((H, W)).astype(np.float32)
    D = np.zeros((3, 4, 1), np.float32)
    D[0, 0, 0] = 1.0
    lam = 0.25
    opt = {"MaxMainIter": 400, "RelStopTol": 1e-9, "NoBndryCross": True,
           "AutoRho": {"Enabled": True}}
    X = O.cbpdn(D, S, lam, opt)[..., 0]
    ref = np.sign(S) * np.maximum(np.abs(S) - np.float32(lam), 0)
    ref[H - 2:, :] = 0.0
    ref[:, W - 3:] = 0.0
    np.testing.assert_allclose(X, ref, atol=1e-6)


def test_projections_leave_the_ams_map_alone():
    """With a mask the impulse map's Y is the AMS step whatever NonNegCoef and
    NoBndryCross say: the masked solve's AMS map keeps negative values and
    values in the boundary band."""
    rng = np.random.default_rng(11)
    H, W, M, K = 16, 16, 2, 3
    D = rng.standard_normal((K, K, M)).astype(np.float32)
    S = rng.standard_normal((H, W)).astype(np.float32)
    Wm = (rng.random((H, W)) < 0.6).astype(np.float32)
    opt = {"MaxMainIter": 40, "RelStopTol": 0.0, "NonNegCoef": True, "NoBndryCross": True,
           "AutoRho": {"Enabled": True}}
    X, info = O.cbpdnmsk(D, S * Wm, Wm, 0.1, opt, return_info=True)
    Y0 = info["Y"][0]
    assert (Y0 < 0).any() and np.abs(Y0[H - 2:, :]).max() > 0
    assert X.min() >= 0.0
    assert np.abs(X[H - 2:, :, :]).max() == 0.0 and np.abs(X[:, W - 2:, :]).max() == 0.0


@pytest.mark.parametrize("variant", ["cbpdn", "cbpdngrd", "cbpdnmsk", "cbpdngrdmsk"])
def test_torch_lean_iterations_equal_numpy_iterations(variant):
    """The multi-threaded torch restatement (the benchmark's CPU baseline and
    relative-error reference) takes the numpy oracle's iterates."""
    from oracle import cbpdn_oracle_torch as OT
    rng = np.random.default_rng(12)
    H, W, M, K = 20, 26, 6, 5
    D = rng.standard_normal((K, K, M)).astype(np.float32)
    S = rng.standard_normal((H, W)).astype(np.float32)
    Wm = (rng.random((H, W)) < 0.7).astype(np.float32)
    opt = {"MaxMainIter": 20, "RelStopTol": 0.0, "AutoRho": {"Enabled": True},
           "NonNegCoef": variant == "cbpdngrd", "NoBndryCross": variant == "cbpdnmsk",
           "GradWeight": np.linspace(0.5, 1.5, M).astype(np.float32)}
    ams = variant.endswith("msk")
    Sx = S * Wm if ams else S
    args = {"cbpdn": (D, Sx, 0.1, opt), "cbpdngrd": (D, Sx, 0.1, 0.3, opt),
            "cbpdnmsk": (D, Sx, Wm, 0.1, opt), "cbpdngrdmsk": (D, Sx, Wm, 0.1, 0.3, opt)}
    X, info = getattr(O, variant)(*args[variant], return_info=True)
    for keep in (False, True):
        Xt, infot = OT.solve(variant, D, Sx, 0.1, opt, mu=0.3, W=Wm if ams else None, chunk=4,
                             keep=keep)
        assert np.linalg.norm(Xt - X) / np.linalg.norm(X) < 1e-11
        np.testing.assert_allclose(infot["hist"]["rho"], info["hist"]["rho"], rtol=1e-12)


def test_torch_chunked_objective_equals_numpy_objective():
    from oracle import cbpdn_oracle_torch as OT
    rng = np.random.default_rng(13)
    D = rng.standard_normal((7, 4, 5))
    S = rng.standard_normal((22, 18))
    Y = rng.standard_normal((7, 22, 18))
    Wm = (rng.random((22, 18)) < 0.6).astype(np.float64)
    wg = rng.random(7)
    for kw in ({}, {"mu": 0.3, "wgrd": wg}, {"mask": Wm}):
        J = O.objective(D, S, Y, 0.2, **kw)
        Jt = OT.objective(D, S, Y, 0.2, chunk=3, **kw)
        assert abs(J - Jt) <= 1e-12 * abs(J)


def test_continued_run_equals_one_run():
    """A run continued from an earlier run's state (the warm start of a
    dictionary-learning outer loop) takes the iterates of one longer run."""
    rng = np.random.default_rng(14)
    D = rng.standard_normal((4, 4, 5)).astype(np.float32)
    S = rng.standard_normal((20, 18)).astype(np.float32)
    opt = {"MaxMainIter": 30, "RelStopTol": 0.0, "AutoRho": {"Enabled": True, "Period": 3}}
    X, info = O.cbpdn(D, S, 0.1, opt, return_info=True)
    _, i1 = O.cbpdn(D, S, 0.1, dict(opt, MaxMainIter=13), return_info=True)
    X2, i2 = O.cbpdn(D, S, 0.1, dict(opt, MaxMainIter=17), return_info=True, start=i1)
    np.testing.assert_array_equal(X2, X)
    assert i2["iterations"] == 30 and i2["rho"] == info["rho"]
