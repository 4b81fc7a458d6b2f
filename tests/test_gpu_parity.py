"""Parity of the CUDA solvers with the compiled reference's outputs (golden
fixtures) and with the FP64 oracle."""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import cases
import sporco_cuda.cbpdn as cb
from oracle import cbpdn_oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_outputs.npz"))

# Relative error bound of the FP32 GPU path against the FP64 oracle: on the
# coefficient maps, and on the functional at them.
REL_TOL = 1e-4
FUNC_TOL = 1e-6
# Small random (unnormalised) dictionaries with adaptive rho amplify float32
# rounding more: the compiled FP32 reference itself is 1.2e-4 from the FP64
# oracle on golden case 15 (32x31, AutoRho).
AUTORHO_TOL = 5e-4


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(1, cases.NCASES + 1))
def test_numpy_path_matches_reference_and_oracle(i):
    c = cases.make_case(i)
    X = cases.run(cb, c)
    Xo = cases.run(O, c)
    assert X.dtype == np.float32 and X.shape == Xo.shape
    # same bound as the reference's own tests (test_cbpdn.py:32,90)
    if i != 19:  # case 19: the reference's U rescale differs (see test_oracle_golden)
        assert O.mse(X, GOLD["case%02d" % i]) < c["tol"]
    tol = AUTORHO_TOL if i in (3, 15) else REL_TOL  # case 3: an unregularised map
    assert _rel(X, Xo) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("i", [1, 4, 6, 11, 14, 16, 19])
def test_torch_path_matches_numpy_path(i):
    c = cases.make_case(i)
    X = cases.run(cb, c)
    ct = dict(c)
    ct["D"] = torch.as_tensor(c["D"], device="cuda")
    ct["S"] = torch.as_tensor(c["S"], device="cuda")
    Xt = cases.run(cb, ct).cpu().numpy()
    assert _rel(Xt, X.astype(np.float64)) < 1e-6


@pytest.mark.gpu
def test_deterministic_bitwise():
    c = cases.make_case(16)
    a = cases.run(cb, c)
    b = cases.run(cb, c)
    assert np.array_equal(a, b)


def _synth(H, W, M, K, density, seed):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((K, K, M))
    D /= np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))
    X0 = (rng.random((H, W, M)) < density) * rng.standard_normal((H, W, M))
    Df = np.fft.rfft2(D, s=(H, W), axes=(0, 1))
    s = np.fft.irfft2(np.sum(Df * np.fft.rfft2(X0, axes=(0, 1)), axis=2), s=(H, W))
    s = s + 0.01 * rng.standard_normal((H, W))
    return D.astype(np.float32), (s - s.mean()).astype(np.float32)


@pytest.mark.gpu
def test_benchmark_shape_256_fixed_rho():
    """256x256, 64 filters 8x8, lambda 0.05, fixed rho: the 200-iteration
    benchmark problem cut to 40 iterations for the FP64 oracle's sake."""
    D, S = _synth(256, 256, 64, 8, 0.01, 12345)
    lam = 0.05
    opt = {"MaxMainIter": 40, "RelStopTol": 0.0, "RelaxParam": 1.8,
           "rho": float(np.float32(50 * np.float32(lam) + 1)), "AutoRho": {"Enabled": False}}
    X = cb.cbpdn(D, S, lam, opt)
    Xo = O.cbpdn(D, S, lam, opt)
    assert _rel(X, Xo) < REL_TOL
    Dm = np.moveaxis(D, 2, 0).astype(np.float64)
    J = O.objective(Dm, S, np.moveaxis(X.astype(np.float64), 2, 0), np.float32(lam))
    Jo = O.objective(Dm, S, np.moveaxis(Xo, 2, 0), np.float32(lam))
    assert abs(J - Jo) / Jo < FUNC_TOL, (J, Jo)


# Column lengths with compiled transform plans and filters of 9..16 rows take
# the convolution column solve with 16 taps (with the gradient term: its
# transform-and-convolution form); 48 rows with 13-row filters wrap the
# circular convolution over more than a quarter of the column; filters of
# 17+ rows take the transform solve.
@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(96, 64, 16), (48, 40, 13), (64, 48, 17), (128, 31, 12)])
@pytest.mark.parametrize("variant", ["cbpdn", "cbpdnmsk", "cbpdngrd"])
def test_column_solve_filter_lengths(shape, variant):
    H, W, K = shape
    D, S = _synth(H, W, 6, K, 0.02, 99)
    lam = 0.05
    opt = {"MaxMainIter": 30, "RelStopTol": 0.0, "RelaxParam": 1.8,
           "rho": float(np.float32(50 * np.float32(lam) + 1)), "AutoRho": {"Enabled": False}}
    if variant == "cbpdn":
        X, Xo = cb.cbpdn(D, S, lam, opt), O.cbpdn(D, S, lam, opt)
    elif variant == "cbpdngrd":
        mu = 0.2
        X, Xo = cb.cbpdngrd(D, S, lam, mu, opt), O.cbpdngrd(D, S, lam, mu, opt)
        assert _rel(X, Xo) < REL_TOL
        _check_functional(D, S, X, Xo, lam, mu=mu, grd=True)
        return
    else:
        Wm = (np.random.default_rng(4).random(S.shape) < 0.7).astype(np.float32)
        X, Xo = cb.cbpdnmsk(D, S * Wm, Wm, lam, opt), O.cbpdnmsk(D, S * Wm, Wm, lam, opt)
    assert _rel(X, Xo) < REL_TOL
    _check_functional(D, S, X, Xo, lam, mask=None if variant == "cbpdn" else Wm)


def _check_functional(D, S, X, Xo, lam, mu=0.0, grd=False, mask=None):
    """The functional at the GPU result against the functional at the FP64
    oracle's result: relative difference at most FUNC_TOL."""
    Dm = np.moveaxis(D, 2, 0).astype(np.float64)
    Sd = S.astype(np.float64) * (mask if mask is not None else 1.0)
    kw = dict(mu=mu, wgrd=np.ones(D.shape[2]) if grd else None, mask=mask)
    J = O.objective(Dm, Sd, np.moveaxis(X.astype(np.float64), 2, 0), np.float32(lam), **kw)
    Jo = O.objective(Dm, Sd, np.moveaxis(np.asarray(Xo, np.float64), 2, 0), np.float32(lam), **kw)
    assert abs(J - Jo) / Jo < FUNC_TOL, (J, Jo)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["cbpdngrd", "cbpdnmsk"])
def test_autorho_128x128(variant):
    """128 x 128, 16 filters 12 x 12, adaptive rho, 30 iterations: the GPU
    result follows the FP64 oracle (the 512 x 512 benchmark shapes are in
    test_gpu_benchmark_shapes.py)."""
    D, S = _synth(128, 128, 16, 12, 0.005, 7)
    lam, mu = 0.05, 0.1
    opt = {"MaxMainIter": 30, "RelStopTol": 0.0, "AutoRho": {"Enabled": True}}
    if variant == "cbpdngrd":
        X = cb.cbpdngrd(D, S, lam, mu, opt)
        Xo = O.cbpdngrd(D, S, lam, mu, opt)
    else:
        W = (np.random.default_rng(3).random(S.shape) < 0.7).astype(np.float32)
        X = cb.cbpdnmsk(D, S * W, W, lam, opt)
        Xo = O.cbpdnmsk(D, S * W, W, lam, opt)
    assert _rel(X, Xo) < REL_TOL
    if variant == "cbpdngrd":
        _check_functional(D, S, X, Xo, lam, mu=mu, grd=True)
    else:
        _check_functional(D, S, X, Xo, lam, mask=W)


@pytest.mark.gpu
def test_early_stopping_iteration_count():
    c = cases.make_case(1)
    opt = dict(c["opt"])
    opt["MaxMainIter"] = 500
    opt["RelStopTol"] = 1e-3
    D = torch.as_tensor(c["D"], device="cuda")
    S = torch.as_tensor(c["S"], device="cuda")
    ds = cb.prepare_device(D.permute(2, 0, 1).contiguous(), S[None], c["lmbda"], opt,
                           check_every=8)
    ds.run()
    it = ds.state()["iterations"][0]
    _, info = O.cbpdn(c["D"], c["S"], c["lmbda"], opt, return_info=True)
    assert it == info["iterations"]


def _uneven_problem():
    rng = np.random.default_rng(11)
    M, K = 6, 5
    D = rng.standard_normal((K, K, M)).astype(np.float32)
    D /= np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))
    shapes = [(32, 31), (24, 40), (32, 31), (48, 48), (24, 40), (31, 17)]
    S_list, W_list = [], []
    for (h, w) in shapes:
        S_list.append(rng.standard_normal((h, w)).astype(np.float32))
        W_list.append((rng.random((h, w)) < 0.7).astype(np.float32))
    S_list = [s * m for s, m in zip(S_list, W_list)]
    lam = rng.uniform(0.05, 0.2, len(shapes)).astype(np.float32)
    return D, S_list, W_list, lam


@pytest.mark.gpu
def test_batched_uneven_sizes_match_oracle():
    """Images of different sizes, per-image masks and lambda, adaptive rho:
    each image follows its own FP64 oracle solve."""
    D, S_list, W_list, lam = _uneven_problem()
    opt = {"MaxMainIter": 60, "RelStopTol": 0.0, "AutoRho": {"Enabled": True}}
    out = cb.cbpdn_batched(D, S_list, lam, opt, W_list=W_list)
    for i in range(len(S_list)):
        Xo = O.cbpdnmsk(D, S_list[i], W_list[i], lam[i], opt)
        assert out[i].shape == Xo.shape
        assert _rel(out[i], Xo) < AUTORHO_TOL, i
        single = cb.cbpdnmsk(D, S_list[i], W_list[i], lam[i], opt)
        assert _rel(out[i], single.astype(np.float64)) < 1e-5, i


@pytest.mark.gpu
def test_batched_early_stopping_per_image():
    """Every image stops on its own test: the batched counts equal those of
    single GPU solves, and the FP64 oracle's within one iteration (the
    stopping decision compares float32-computed residuals with 1e-3)."""
    D, S_list, W_list, lam = _uneven_problem()
    opt = {"MaxMainIter": 300, "RelStopTol": 2e-3, "AutoRho": {"Enabled": True}}
    out, iters = cb.cbpdn_batched(D, S_list, lam, opt, W_list=W_list, return_info=True)
    assert min(iters) < 300 and len(set(iters)) > 1  # images stop on their own
    for i in range(len(S_list)):
        Dt = torch.as_tensor(D, device="cuda")
        St = torch.as_tensor(S_list[i], device="cuda")
        Wt = torch.as_tensor(W_list[i], device="cuda")
        single, it1 = cb.cbpdn_batched(Dt, [St], lam[i:i + 1], opt, W_list=[Wt],
                                       return_info=True)
        assert iters[i] == it1[0]
        assert _rel(out[i], single[0].cpu().numpy().astype(np.float64)) < 1e-5
        _, info = O.cbpdnmsk(D, S_list[i], W_list[i], lam[i], opt, return_info=True)
        assert abs(iters[i] - info["iterations"]) <= 1, (iters[i], info["iterations"])


@pytest.mark.gpu
def test_batched_equals_single_solves():
    rng = np.random.default_rng(12)
    D = rng.standard_normal((4, 4, 5)).astype(np.float32)
    S_list = [rng.standard_normal((40, 36)).astype(np.float32) for _ in range(3)]
    opt = {"MaxMainIter": 30, "RelStopTol": 0.0, "AutoRho": {"Enabled": False}}
    out = cb.cbpdn_batched(D, S_list, 0.1, opt)
    for s, X in zip(S_list, out):
        assert np.array_equal(X, cb.cbpdn(D, s, 0.1, opt))


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["cbpdn", "cbpdngrd"])
def test_device_functional_matches_oracle(variant):
    """The functional the solver records per iteration on the device (the
    Verbose statistics, at Y) against the FP64 functional at the returned Y:
    data fidelity, L1 term and total at the last iteration."""
    grd = variant == "cbpdngrd"
    D, S = _synth(64, 48, 6, 8, 0.02, 5)
    lam, mu = 0.05, 0.1
    opt = {"MaxMainIter": 12, "RelStopTol": 0.0, "AutoRho": {"Enabled": True}}
    Dm = np.moveaxis(D, 2, 0).copy()
    ds = cb.prepare_device(torch.tensor(Dm, device="cuda"), torch.tensor(S, device="cuda")[None],
                           lam, opt, mu=mu if grd else 0.0, grd=grd, record_itstat=True)
    Y = ds.run()[0].double().cpu().numpy()
    st = ds.state()
    k = st["iterations"][0]
    J, Jdf, Jl1 = st["itstat"][0, k - 1, 5:8]
    D64, S64 = Dm.astype(np.float64), S.astype(np.float64)
    kw = dict(mu=mu, wgrd=np.ones(Dm.shape[0])) if grd else {}
    Jo = O.objective(D64, S64, Y, np.float32(lam), **kw)
    Jdfo = O.objective(D64, S64, Y, 0.0)
    assert abs(Jdf - Jdfo) / Jdfo < 1e-5, (Jdf, Jdfo)
    assert abs(Jl1 - np.sum(np.abs(Y))) / np.sum(np.abs(Y)) < 1e-6
    assert abs(J - Jo) / Jo < 1e-5, (J, Jo)


@pytest.mark.gpu
def test_verbose_table(capfd):
    """Verbose solves through the reference-compatible C ABI print the
    reference's table: one row per iteration, functional columns included."""
    c = cases.make_case(1)
    opt = dict(c["opt"], Verbose=True, MaxMainIter=7)
    cb.cbpdn(c["D"], c["S"], c["lmbda"], opt)
    out = capfd.readouterr().out.splitlines()
    assert out[0].split()[:4] == ["Itn", "Fnc", "DFid", "Regl1"]
    rows = [l for l in out if l[:4].strip().isdigit()]
    assert len(rows) == 7
    fnc = [float(r.split()[1]) for r in rows]
    assert all(np.isfinite(fnc)) and fnc[-1] > 0


@pytest.mark.gpu
def test_cancel_stops_a_running_solve():
    """sc_cancel from another thread stops a long fixed-iteration solve at its
    next chunk: SolverError with SC_ERR_CANCELLED, well before the end; a solve
    started afterwards runs normally."""
    import threading
    import time
    from sporco_cuda import _lib
    D, S = _synth(512, 512, 32, 8, 0.01, 3)
    opt = {"MaxMainIter": 20000, "RelStopTol": 0.0, "AutoRho": {"Enabled": False}}
    Dm = torch.tensor(np.moveaxis(D, 2, 0).copy(), device="cuda")
    St = torch.tensor(S, device="cuda")[None]
    ds = cb.prepare_device(Dm, St, 0.05, opt, check_every=16)
    ds.run()  # set-up and autotuning out of the way (the run is the full solve)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ds.run()
    torch.cuda.synchronize()
    full = time.perf_counter() - t0
    err = {}

    def work():
        try:
            ds.run()
        except _lib.SolverError as e:
            err["e"] = e
    th = threading.Thread(target=work)
    t0 = time.perf_counter()
    th.start()
    time.sleep(0.1 * full)
    _lib.sc_cancel()
    th.join()
    took = time.perf_counter() - t0
    assert "e" in err and err["e"].status == 7, err
    assert took < 0.6 * full, (took, full)
    ds.run()  # a new solve is not cancelled
