"""Argument checks of the Python mirror (multifloats_b200.api) that run before
any GPU work: wrong sizes and unusable output buffers raise ValueError instead
of letting the library write past a buffer or dereference a host pointer on
the device."""
import numpy as np
import pytest

from multifloats_b200 import api


def test_host_output_buffers_are_checked():
    a, b = np.zeros(2 * 6), np.zeros(2 * 6)
    for bad in (np.zeros(3), np.zeros(8, dtype=np.float32), np.zeros(16)[::2], [0.0] * 8):
        with pytest.raises(ValueError):
            api.matmuldd_mm(a, b, 2, 3, 2, out=bad)
    with pytest.raises(ValueError):
        api.exp(np.zeros(2 * 5), out=np.zeros(2 * 4))
    with pytest.raises(ValueError):
        api.sincos(np.zeros(2 * 5), s=np.zeros(2 * 5), c=np.zeros(2 * 6))


def test_operand_sizes_are_checked():
    with pytest.raises(ValueError):
        api.matmuldd_mm(np.zeros(2 * 5), np.zeros(2 * 6), 2, 3, 2)
    with pytest.raises(ValueError):
        api.matmuldd_mm_crt(np.zeros(2 * 6), np.zeros(2 * 7), 2, 3, 2)
    with pytest.raises(ValueError):  # host calls have the fixed target 8
        api.matmuldd_mm_crt(np.zeros(2 * 6), np.zeros(2 * 6), 2, 3, 2, target=2.0)


def test_wait_limit_setter_round_trip():
    """mfcuda_set_wait_limit_ns returns the previous setting (0 = the 2 s
    default) and touches no device."""
    from multifloats_b200 import _lib

    L = _lib.lib()
    prev = L.mfcuda_set_wait_limit_ns(12345)
    try:
        assert L.mfcuda_set_wait_limit_ns(777) == 12345
    finally:
        assert L.mfcuda_set_wait_limit_ns(prev) == 777
