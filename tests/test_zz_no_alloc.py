"""sc_rfft2_noalloc: the 2-D real FFT for callers that must not allocate
device memory (its twiddle scratch is a static device array of the library).

Checked through the C ABI against sc_rfft2, the entry point that takes its
scratch from the allocator, on two calls in a row with different sizes, so
that the second call runs on scratch the first one left behind.  This file
is collected last on purpose.
"""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from sporco_cuda import _lib

# same bound as the FFT tests in test_gpu_fft.py
TOL = 2e-6


def _call(fn, x):
    count, H, W = x.shape
    xt = torch.as_tensor(x, device="cuda")
    out = torch.zeros((count, H, W // 2 + 1), dtype=torch.complex64, device="cuda")
    st = fn(C.c_void_p(xt.data_ptr()), C.c_void_p(out.data_ptr()), count, H, W,
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_rfft2_matches_allocating_entry_point_twice():
    rng = np.random.default_rng(2024)
    for H, W in ((512, 384), (32, 31)):
        x = rng.standard_normal((3, H, W)).astype(np.float32)
        got = _call(_lib.sc_rfft2_noalloc, x)
        ref = _call(_lib.sc_rfft2, x)
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err < TOL, (H, W, err)
        exact = np.fft.rfft2(x.astype(np.float64))
        assert np.linalg.norm(got - exact) / np.linalg.norm(exact) < TOL


@pytest.mark.gpu
def test_allocating_entry_points_still_work_after_noalloc():
    """A call at a small size with no compile-time plan, then the allocating
    transform at larger sizes with none (their kernels need more shared
    memory than the small call did): both still run and match numpy."""
    rng = np.random.default_rng(7)
    for (h0, w0), (H, W) in (((32, 31), (500, 300)), ((20, 27), (333, 601))):
        x0 = rng.standard_normal((2, h0, w0)).astype(np.float32)
        got0 = _call(_lib.sc_rfft2_noalloc, x0)
        ex0 = np.fft.rfft2(x0.astype(np.float64))
        assert np.linalg.norm(got0 - ex0) / np.linalg.norm(ex0) < TOL
        x = rng.standard_normal((2, H, W)).astype(np.float32)
        got = _call(_lib.sc_rfft2, x)
        exact = np.fft.rfft2(x.astype(np.float64))
        assert np.linalg.norm(got - exact) / np.linalg.norm(exact) < TOL, (H, W)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    st = _lib.sc_rfft2_noalloc(C.c_void_p(1), C.c_void_p(1), 1, 4096, 8192, None)
    assert st == 2  # SC_ERR_UNSUPPORTED
    assert b"static scratch" in _lib.sc_last_error()
