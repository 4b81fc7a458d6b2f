"""Two host threads driving the library at once on one GPU: each solve keeps
its state in its own workspace, and the process-wide caches (kernel
attributes, occupancy answers, autotuned cluster sizes, FFT-tool twiddle
tables) are shared under a lock.  Results must equal the single-thread
results bit for bit."""

import ctypes as C
import threading

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import sporco_cuda.cbpdn as cb
from sporco_cuda import _lib


def _problem(H, W, M, K, seed):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((K, K, M)).astype(np.float32)
    S = rng.standard_normal((H, W)).astype(np.float32)
    return D, S


OPT = {"MaxMainIter": 40, "RelStopTol": 0.0, "AutoRho": {"Enabled": True}}
# the convolution column solve at compiled lengths; the transform solve at
# generic lengths; a gradient problem
PROBLEMS = [(_problem(96, 64, 6, 12, 1), "cbpdn"), (_problem(72, 50, 5, 7, 2), "cbpdn"),
            (_problem(128, 96, 4, 9, 3), "cbpdngrd")]


def _solve_torch(i):
    (D, S), variant = PROBLEMS[i]
    Dt, St = torch.tensor(D, device="cuda"), torch.tensor(S, device="cuda")
    if variant == "cbpdngrd":
        return cb.cbpdngrd(Dt, St, 0.05, 0.1, OPT).cpu().numpy()
    return cb.cbpdn(Dt, St, 0.05, OPT).cpu().numpy()


def _solve_numpy(i):
    (D, S), variant = PROBLEMS[i]
    if variant == "cbpdngrd":
        return cb.cbpdngrd(D, S, 0.05, 0.1, OPT)
    return cb.cbpdn(D, S, 0.05, OPT)


def _rfft2(x, H, W):
    xt = torch.as_tensor(x, device="cuda")
    out = torch.empty((x.shape[0], H, W // 2 + 1), dtype=torch.complex64, device="cuda")
    _lib.check(_lib.sc_rfft2(C.c_void_p(xt.data_ptr()), C.c_void_p(out.data_ptr()), x.shape[0],
                             H, W, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.current_stream().synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
def test_two_host_threads_solve_at_once_bitwise():
    # single-thread results first (they also settle the autotuner's choice of
    # cluster size for these shapes, which both runs then share)
    ref_t = [_solve_torch(i) for i in range(len(PROBLEMS))]
    ref_n = [_solve_numpy(i) for i in range(len(PROBLEMS))]
    rng = np.random.default_rng(9)
    # FFT sizes no earlier call used: both threads create twiddle tables
    fft_in = [rng.standard_normal((2, 37, 53)).astype(np.float32),
              rng.standard_normal((2, 41, 29)).astype(np.float32)]
    fft_ref = [np.fft.rfft2(x.astype(np.float64)) for x in fft_in]
    out = {}
    errors = []
    barrier = threading.Barrier(2)

    def work(tid):
        try:
            with torch.cuda.stream(torch.cuda.Stream()):
                barrier.wait()
                for rep in range(3):
                    for i in range(len(PROBLEMS)):
                        j = (i + tid) % len(PROBLEMS)
                        out[(tid, rep, "t", j)] = _solve_torch(j)
                        out[(tid, rep, "n", j)] = _solve_numpy(j)
                    x = fft_in[(tid + rep) % 2]
                    out[(tid, rep, "f")] = (_rfft2(x, *x.shape[1:]), (tid + rep) % 2)
        except Exception as e:  # reported below
            errors.append(e)

    th = [threading.Thread(target=work, args=(t,)) for t in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    for key, val in out.items():
        if key[2] == "t":
            assert np.array_equal(val, ref_t[key[3]]), key
        elif key[2] == "n":
            assert np.array_equal(val, ref_n[key[3]]), key
        else:
            got, which = val
            ex = fft_ref[which]
            assert np.linalg.norm(got - ex) / np.linalg.norm(ex) < 2e-6, key
