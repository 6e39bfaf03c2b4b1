"""The allocation-free converting upload, dgk_convert_upload_noalloc, against the runner's own converting
upload (dgk_copy_to_device with a float64 -> float32 binding).

Callers that may not allocate device memory once running -- a host application that owns the device-memory
budget, or a time-stepping loop that cannot absorb a cudaMalloc -- use the allocation-free entry point, which
stages through a fixed 8 MiB array in the library's device image.  The two paths must write identical device
data (the conversion is exact, so the tolerance is zero), on two calls in a row, and sizes beyond the fixed
array must be refused.  This file is collected last so that a stop-at-first-failure run has run every other
test before it.  The refusal of an oversized count happens before any device work, so it is also checked
without a GPU.
"""
import ctypes

import numpy as np
import pytest

import dgkernel_b200 as d
from dgkernel_b200 import _lib
from dgkernel_b200.runner import Config, Float32, Input, Runner


def test_noalloc_refuses_wrapping_count_without_device_work():
    # count * 8 wraps to 0 in 64 bits; the size check must refuse it before any copy or launch
    L = _lib.lib()
    buf = np.zeros(4)
    p = ctypes.c_void_p(buf.ctypes.data)
    for count in (1 << 61, (1 << 63) - 1, (8 << 20) // 8 + 1):
        assert L.dgk_convert_upload_noalloc(p, d.Float64, p, d.Float32, count, None) == _lib.ERR_INVALID
        assert b"8 MiB" in L.dgk_global_error()


@pytest.mark.gpu
def test_noalloc_upload_matches_runner_upload_twice():
    n = 300_000
    r = Runner(Config(K=[n]))
    r.DefineBindings(Input("A").Bind(np.zeros(n)).DeviceMemType(Float32),
                     Input("B").Bind(np.zeros(n)).DeviceMemType(Float32))
    r.AllocateDevice()
    dst = ctypes.c_void_p(r.DevicePtr("B"))
    L = _lib.lib()
    rng = np.random.default_rng(11)
    for call in range(2):
        host = np.ascontiguousarray(rng.standard_normal(n) * 10.0 ** (3 * call))
        r.CopyToDevice("A", host)  # the existing entry point
        _lib.check(L.dgk_convert_upload_noalloc(ctypes.c_void_p(host.ctypes.data), d.Float64, dst, d.Float32, n,
                                                None))
        a = r.CopyPartitionToHost("A", 0)
        got = r.CopyPartitionToHost("B", 0)
        assert np.array_equal(got, a)
        assert np.array_equal(got, host.astype(np.float32))
    big = np.zeros((8 << 20) // 8 + 1)
    rc = L.dgk_convert_upload_noalloc(ctypes.c_void_p(big.ctypes.data), d.Float64, dst, d.Float32, big.size, None)
    assert rc == _lib.ERR_INVALID
    assert b"8 MiB" in L.dgk_global_error()
    r.Free()
