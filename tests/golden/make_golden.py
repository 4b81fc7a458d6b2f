"""Generate tests/golden/ref_outputs.npz from the compiled reference.

Runs the reference's own FP32 GPU solvers (built from the reference sources
by ``make -C oracle ref`` into ``oracle/_ref/libsporco_cuda_ref.so``) on every
case of ``tests/golden/cases.py`` and stores their outputs.  Needs a GPU; it
is run once on the GPU host and its (small) output is committed:

    python tests/golden/make_golden.py [output.npz]

The inputs are not stored: ``cases.make_case`` regenerates them bit for bit
from their seeds.
"""

from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import cases  # noqa: E402
from oracle import cbpdn_oracle, ref_abi  # noqa: E402


def main(path=None):
    out = {}
    for i in range(1, cases.NCASES + 1):
        c = cases.make_case(i)
        X = cases.run(ref_abi, c)
        Xo = cases.run(cbpdn_oracle, c)
        out["case%02d" % i] = np.asarray(X, dtype=np.float32)
        rel = np.linalg.norm(X - Xo) / max(np.linalg.norm(Xo), 1e-30)
        print("case %2d %-12s mse(ref, oracle)=%.3e rel=%.3e" % (
            i, c["kind"], cbpdn_oracle.mse(X, Xo), rel), flush=True)
    if path is None:
        path = os.path.join(ROOT, "tests", "golden", "ref_outputs.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
