"""The hand-written Stockham R2C / C2R transforms against numpy (FP64)."""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from sporco_cuda import _lib

SIZES = [(32, 31), (31, 32), (64, 64), (24, 40), (7, 13), (1, 8), (8, 1), (1, 1),
         (256, 256), (192, 384), (128, 768), (512, 512), (61, 97), (2048, 64), (64, 2048),
         (25, 1000), (2048, 2048)]


def _rfft2_gpu(x):
    count, H, W = x.shape
    xt = torch.as_tensor(x, device="cuda")
    out = torch.empty((count, H, W // 2 + 1), dtype=torch.complex64, device="cuda")
    st = _lib.sc_rfft2(C.c_void_p(xt.data_ptr()), C.c_void_p(out.data_ptr()), count, H, W,
                       C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st)
    return out.cpu().numpy()


def _irfft2_gpu(xf, H, W):
    count = xf.shape[0]
    xt = torch.as_tensor(xf, device="cuda")
    out = torch.empty((count, H, W), dtype=torch.float32, device="cuda")
    st = _lib.sc_irfft2(C.c_void_p(xt.data_ptr()), C.c_void_p(out.data_ptr()), count, H, W,
                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st)
    return out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("H,W", SIZES)
def test_rfft2_matches_numpy(H, W):
    rng = np.random.default_rng(H * 10007 + W)
    count = 3 if H * W < 1 << 20 else 1
    x = rng.standard_normal((count, H, W)).astype(np.float32)
    ref = np.fft.rfft2(x.astype(np.float64))
    got = _rfft2_gpu(x)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 2e-6, err


@pytest.mark.gpu
@pytest.mark.parametrize("H,W", SIZES)
def test_irfft2_roundtrip(H, W):
    rng = np.random.default_rng(H * 31 + W)
    x = rng.standard_normal((2, H, W)).astype(np.float32)
    xf = np.fft.rfft2(x.astype(np.float64)).astype(np.complex64)
    got = _irfft2_gpu(xf, H, W)
    ref = np.fft.irfft2(xf.astype(np.complex128), s=(H, W))
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 2e-6, err
