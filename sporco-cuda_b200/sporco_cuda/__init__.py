"""B200 (sm_100a) drop-in for ``sporco_cuda``: ADMM convolutional sparse
coding solvers (cbpdn, cbpdnmsk, cbpdngrd, cbpdngrdmsk) on hand-written CUDA
kernels, with the reference's Python signatures and option dicts."""

from __future__ import absolute_import

__version__ = '0.0.6b1+b200.0.1'

from . import util  # noqa: E402,F401
from . import cbpdn  # noqa: E402,F401
