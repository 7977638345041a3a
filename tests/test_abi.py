"""The C ABI without a GPU: the library loads, exports every declared symbol,
and validates input before touching CUDA."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from gpumetropolis_b200 import _native
from gpumetropolis_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"\b(gpum_b200_\w+)\s*\(", src))
    return names


@pytest.fixture(scope="module")
def lib():
    build()
    return C.CDLL(_native.LIB_PATH)


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 15
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert set(_native.SIGNATURES) >= names


def test_version_and_no_device_on_cpu_host(native):
    assert b"sm_100a" in native.load().gpum_b200_version()
    if not os.path.exists("/dev/nvidia0"):
        assert native.available() is False


def test_validate_program(native):
    assert native.validate_program([1, 0, 0, 0, 3, 0], 1, 1, 0) == 2
    bad = [
        ([1, 0, 3], 1, 1, 0),              # odd length
        ([3, 0], 0, 1, 0),                 # underflow
        ([0, 5], 1, 1, 0),                 # constant out of range
        ([1, 3], 0, 1, 0),                 # parameter out of range
        ([2, 1], 0, 1, 1),                 # column out of range
    ]
    for code, nc, npar, ncol in bad:
        with pytest.raises(native.GpumError) as e:
            native.validate_program(code, nc, npar, ncol)
        assert e.value.code == native.ERR_INVALID
    with pytest.raises(native.GpumError):  # a prior may not read data
        native.validate_program([2, 0], 0, 1, 1, allow_data=False)
    deep = [1, 0] * 33 + [3, 0] * 32
    with pytest.raises(native.GpumError):
        native.validate_program(deep, 0, 1, 0)


def test_entry_points_reject_bad_input_before_cuda(native):
    # malformed bytecode is an argument error, whatever the machine has
    with pytest.raises(native.GpumError) as e:
        native.loglik_batch([3, 0], [], 1, np.zeros(2), 1, 2, [0.0])
    assert e.value.code == native.ERR_INVALID
    with pytest.raises(native.GpumError) as e:
        native.Session([1, 7], [], [], [], 1, np.zeros(2), 1, 2)
    assert e.value.code == native.ERR_INVALID
    with pytest.raises(native.GpumError) as e:
        native.Session([1, 0], [], [2, 0], [], 1, np.zeros(2), 1, 2)  # prior reads data
    assert e.value.code == native.ERR_INVALID
    if not os.path.exists("/dev/nvidia0"):
        with pytest.raises(native.GpumError) as e:
            native.loglik_batch([1, 0], [], 1, np.zeros(2), 1, 2, [0.0])
        assert e.value.code == native.ERR_NODEVICE


def test_output_buffers_are_checked_before_any_call():
    # caller-provided draws buffers (Session.run / run_da / run out_draws)
    # must be contiguous 1-D float32 arrays of at least the draws' size
    from gpumetropolis_b200._native import _out_f32
    buf = np.zeros(12, np.float32)
    assert _out_f32(buf, 12) is buf
    assert _out_f32(None, 0).size == 1
    for bad in (np.zeros(11, np.float32), np.zeros(12, np.float64),
                np.zeros((3, 4), np.float32), np.zeros(24, np.float32)[::2]):
        with pytest.raises(ValueError, match="out_draws"):
            _out_f32(bad, 12)
