"""Device queries, as the reference's sporco_cuda/tests/test_util.py:8-25."""

import pytest

import sporco_cuda.util as cu


def test_device_count():
    assert cu.device_count() >= 0


@pytest.mark.gpu
def test_current_device():
    assert cu.current_device() >= 0
    assert cu.current_device(0) == 0


@pytest.mark.gpu
def test_memory_info():
    f, t = cu.memory_info()
    assert f >= 0 and t > 0


@pytest.mark.gpu
def test_device_name():
    nm = cu.device_name()
    assert nm is not None and nm != ''
