"""Device queries, as ``sporco_cuda.util`` (sporco_cuda/util.pyx:10-45)."""

from __future__ import annotations

import ctypes as C

from . import _lib

__all__ = ["device_count", "current_device", "memory_info", "device_name"]


def device_count():
    """Number of CUDA devices (util.pyx:10-12)."""
    return _lib.get_device_count()


def current_device(newdev=None):
    """Get, and optionally first set, the current device (util.pyx:15-27)."""
    dev = C.c_int(0)
    if newdev is not None:
        err = _lib.set_current_device(int(newdev))
        if err != 0:
            raise RuntimeError('CUDA error %d while setting device' % err)
    err = _lib.get_current_device(C.byref(dev))
    if err != 0:
        raise RuntimeError('CUDA error %d while getting current device' % err)
    return dev.value


def memory_info():
    """(free, total) device memory in bytes (util.pyx:30-36)."""
    free, total = C.c_size_t(0), C.c_size_t(0)
    err = _lib.get_memory_info(C.byref(free), C.byref(total))
    if err != 0:
        raise RuntimeError('CUDA error %d' % err)
    return free.value, total.value


def device_name(dev=0):
    """Name of a device, or None (util.pyx:39-45)."""
    s = _lib.get_device_name(int(dev))
    return None if s is None else s.decode('UTF-8')
