"""Launch options read from the environment at the first solve of a process
(so each case runs in a child process): programmatic dependent launch
(SPORCO_B200_PDL=1) and a fixed column-pass cluster size
(SPORCO_B200_COL_CLUSTER).  Both change only how the kernels are launched;
the results must match the FP64 oracle as the default launches do."""

import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import cbpdn_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
import numpy as np
sys.path[:0] = [{root!r}, {pkg!r}]
import sporco_cuda.cbpdn as cb
d = np.load({inp!r})
opt = {{"MaxMainIter": 30, "RelStopTol": 0.0, "AutoRho": {{"Enabled": True}}}}
if d["variant"] == "cbpdngrd":
    X = cb.cbpdngrd(d["D"], d["S"], 0.05, 0.1, opt)
else:
    X = cb.cbpdn(d["D"], d["S"], 0.05, opt)
np.save({out!r}, X)
"""


def _synth(H, W, M, K, seed):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((K, K, M))
    D /= np.sqrt(np.sum(D * D, axis=(0, 1), keepdims=True))
    X0 = (rng.random((H, W, M)) < 0.01) * rng.standard_normal((H, W, M))
    Df = np.fft.rfft2(D, s=(H, W), axes=(0, 1))
    s = np.fft.irfft2(np.sum(Df * np.fft.rfft2(X0, axes=(0, 1)), axis=2), s=(H, W))
    s = s + 0.01 * rng.standard_normal((H, W))
    return D.astype(np.float32), (s - s.mean()).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("env", [{"SPORCO_B200_PDL": "1"},
                                 {"SPORCO_B200_COL_CLUSTER": "2"},
                                 {"SPORCO_B200_PDL": "1", "SPORCO_B200_COL_CLUSTER": "4"}])
@pytest.mark.parametrize("variant", ["cbpdn", "cbpdngrd"])
def test_launch_options_keep_results(tmp_path, env, variant):
    D, S = _synth(128, 96, 12, 12, 5)
    inp = str(tmp_path / "in.npz")
    out = str(tmp_path / "out.npy")
    np.savez(inp, D=D, S=S, variant=variant)
    code = CHILD.format(root=ROOT, pkg=os.path.join(ROOT, "sporco-cuda_b200"), inp=inp, out=out)
    r = subprocess.run([sys.executable, "-c", code], env=dict(os.environ, **env),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    X = np.load(out)
    opt = {"MaxMainIter": 30, "RelStopTol": 0.0, "AutoRho": {"Enabled": True}}
    Xo = O.cbpdngrd(D, S, 0.05, 0.1, opt) if variant == "cbpdngrd" else O.cbpdn(D, S, 0.05, opt)
    rel = np.linalg.norm(X.astype(np.float64) - Xo) / np.linalg.norm(Xo)
    assert rel < 1e-4, rel
