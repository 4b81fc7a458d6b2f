"""Column-pass variants the autotuner chooses between: tiles of 4 or 2
columns and, at column lengths 512-1024, the radix-16 or radix-8 column
plan.  A variant changes only how the work is split over threads and CTAs:
at one cluster size every variant sums the maps and filter taps in the same
order, so the coefficient maps must agree bit for bit between tile widths,
and every variant must agree with the FP64 oracle.

Each case runs in a child process, the variant fixed by the launch options
SPORCO_B200_COL_TILE, SPORCO_B200_COL_RADIX and SPORCO_B200_COL_CLUSTER
(which also keeps the autotuner off)."""

import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import cbpdn_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REL_TOL = 1e-4

CHILD = r"""
import sys
import numpy as np
sys.path[:0] = [{root!r}, {pkg!r}]
import sporco_cuda.cbpdn as cb
d = np.load({inp!r})
opt = {{"MaxMainIter": int(d["iters"]), "RelStopTol": 0.0, "RelaxParam": 1.8, "rho": None,
        "AutoRho": {{"Enabled": True, "Period": 1, "Scaling": 1000.0, "RsdlRatio": 1.2,
                     "AutoScaling": True}}}}
v = str(d["variant"])
if v == "cbpdngrd":
    X = cb.cbpdngrd(d["D"], d["S"], 0.05, 0.1, opt)
elif v == "cbpdnmsk":
    X = cb.cbpdnmsk(d["D"], d["S"] * d["W"], d["W"], 0.05, opt)
else:
    X = cb.cbpdn(d["D"], d["S"], 0.05, opt)
np.save({out!r}, X)
"""


def _synth(H, W, M, K, seed):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((K, K, M))
    D /= np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))
    X0 = (rng.random((H, W, M)) < 0.005) * rng.standard_normal((H, W, M))
    Df = np.fft.rfft2(D, s=(H, W), axes=(0, 1))
    s = np.fft.irfft2(np.sum(Df * np.fft.rfft2(X0, axes=(0, 1)), axis=2), s=(H, W))
    s = s + 0.01 * rng.standard_normal((H, W))
    return D.astype(np.float32), (s - s.mean()).astype(np.float32)


def _run(tmp_path, tag, env, D, S, W, variant, iters):
    inp = str(tmp_path / f"in_{tag}.npz")
    out = str(tmp_path / f"out_{tag}.npy")
    np.savez(inp, D=D, S=S, W=W, variant=variant, iters=iters)
    code = CHILD.format(root=ROOT, pkg=os.path.join(ROOT, "sporco-cuda_b200"), inp=inp, out=out)
    r = subprocess.run([sys.executable, "-c", code], env=dict(os.environ, **env),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(out)


def _oracle(D, S, W, variant, iters):
    opt = {"MaxMainIter": iters, "RelStopTol": 0.0, "RelaxParam": 1.8, "rho": None,
           "AutoRho": {"Enabled": True, "Period": 1, "Scaling": 1000.0, "RsdlRatio": 1.2,
                       "AutoScaling": True}}
    if variant == "cbpdngrd":
        return O.cbpdngrd(D, S, 0.05, 0.1, opt)
    if variant == "cbpdnmsk":
        return O.cbpdnmsk(D, S * W, W, 0.05, opt)
    return O.cbpdn(D, S, 0.05, opt)


# (size, maps, filter size, solve, column radix, cluster size, iterations):
# the convolution solves C8 (8 x 8 filters), C16 (12 x 12, 16 x 16) and the
# gradient solve G16, at the radix-16 plans of 512 / 1024 / 2048 and the
# radix-8 plans of 512 / 1024
CASES = [
    (512, 24, 12, "cbpdngrd", 16, 4, 20),
    (512, 24, 12, "cbpdnmsk", 8, 4, 20),
    (512, 24, 8, "cbpdn", 8, 3, 20),
    (1024, 16, 16, "cbpdn", 16, 2, 10),
    (1024, 16, 12, "cbpdngrd", 8, 4, 10),
    (2048, 8, 16, "cbpdn", 16, 2, 6),
]


@pytest.mark.gpu
@pytest.mark.parametrize("size,M,K,variant,rm,G,iters", CASES)
def test_tile_widths_agree_bitwise_and_with_oracle(tmp_path, size, M, K, variant, rm, G, iters):
    D, S = _synth(size, size, M, K, 100 + size + K)
    W = (np.random.default_rng(7).random(S.shape) < 0.7).astype(np.float32)
    base = {"SPORCO_B200_COL_CLUSTER": str(G), "SPORCO_B200_COL_RADIX": str(rm)}
    X4 = _run(tmp_path, "t4", dict(base, SPORCO_B200_COL_TILE="4"), D, S, W, variant, iters)
    X2 = _run(tmp_path, "t2", dict(base, SPORCO_B200_COL_TILE="2"), D, S, W, variant, iters)
    assert np.array_equal(X2, X4), np.abs(X2.astype(np.float64) - X4).max()
    Xo = _oracle(D, S, W, variant, iters)
    rel = np.linalg.norm(X2.astype(np.float64) - Xo) / np.linalg.norm(Xo)
    assert rel < REL_TOL, rel


SPLIT_CHILD = r"""
import sys
import numpy as np
sys.path[:0] = [{root!r}, {pkg!r}]
import sporco_cuda.cbpdn as cb
d = np.load({inp!r})
opt = {{"MaxMainIter": int(d["iters"]), "RelStopTol": 0.0, "RelaxParam": 1.8, "rho": None,
        "AutoRho": {{"Enabled": True, "Period": 1, "Scaling": 1000.0, "RsdlRatio": 1.2,
                     "AutoScaling": True}}}}
singles = [cb.cbpdn(d["D"], s, 0.05, opt) for s in (d["S0"], d["S1"])]
batch = cb.cbpdn_batched(d["D"], [d["S0"], d["S1"]], 0.05, opt)
np.savez({out!r}, X0=singles[0], X1=singles[1], B0=batch[0], B1=batch[1])
"""


@pytest.mark.gpu
def test_tail_split_batch_equals_single_and_oracle(tmp_path):
    """2048 x 2048 with clusters of 2: 257 column tiles fill three rounds of
    the 74 resident clusters and part of a fourth, whose 35 tiles the split
    runs as a second launch with clusters of 3.  A batch of two images is
    split at the same tile, so it equals the two single solves bit for bit;
    both agree with the FP64 oracle."""
    D, S0 = _synth(2048, 2048, 8, 16, 301)
    _, S1 = _synth(2048, 2048, 8, 16, 302)
    iters = 6
    inp = str(tmp_path / "in.npz")
    out = str(tmp_path / "out.npz")
    np.savez(inp, D=D, S0=S0, S1=S1, iters=iters)
    code = SPLIT_CHILD.format(root=ROOT, pkg=os.path.join(ROOT, "sporco-cuda_b200"), inp=inp,
                              out=out)
    env = dict(os.environ, SPORCO_B200_COL_CLUSTER="2", SPORCO_B200_COL_SPLIT="3")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    o = np.load(out)
    assert np.array_equal(o["X0"], o["B0"]) and np.array_equal(o["X1"], o["B1"])
    Xo = _oracle(D, S0, None, "cbpdn", iters)
    rel = np.linalg.norm(o["X0"].astype(np.float64) - Xo) / np.linalg.norm(Xo)
    assert rel < REL_TOL, rel
