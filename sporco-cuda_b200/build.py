"""Build the sm_100a shared library libsporco_b200.so in place.

    python sporco-cuda_b200/build.py [--force] [-j N]

Compiles every .cu under csrc/ with nvcc for sm_100a into an object of its
own (in parallel; the kernel instantiations are spread over several
translation units for that reason) and links them into
sporco_cuda/libsporco_b200.so, next to the Python package that loads it.
Objects are kept in _build/ and rebuilt when their source or any header is
newer.
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "sporco_cuda", "libsporco_b200.so")
INC = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", *ARCH,
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
    "-I" + CSRC, "-I" + INC,
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + \
        sorted(glob.glob(os.path.join(INC, "*.h")))


def _obj(src):
    return os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def up_to_date():
    return os.path.exists(OUT) and not _newer(OUT, sources() + headers())


def build(force=False, verbose=False, jobs=None):
    if not force and up_to_date():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    hdrs = headers()
    todo = [s for s in sources() if force or _newer(_obj(s), [s] + hdrs)]

    def compile_one(src):
        cmd = [nvcc] + NVCC_FLAGS + ["-c", src, "-o", _obj(src)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        return src

    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(jobs) as ex:
        for f in cf.as_completed([ex.submit(compile_one, s) for s in todo]):
            f.result()
    cmd = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC"] + [_obj(s) for s in sources()] + \
        ["-o", OUT]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    j = None
    if "-j" in sys.argv:
        j = int(sys.argv[sys.argv.index("-j") + 1])
    print(build(force="--force" in sys.argv, verbose=True, jobs=j))
