"""Runner planning on the host (no device): offsets, binding errors, kernel signatures, the preamble, and the
C-ABI exports.  Mirrors runner/runner_test.go:103-180, 474-537 and runner/binding_test.go:315-367."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import dgkernel_b200 as d
from dgkernel_b200 import _lib
from dgkernel_b200.runner import Config, Input, Output, InOut, Scalar, Temp, Runner
from oracle import gonudg_ref as g

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def host_runner(K, **kw):
    return Runner(Config(K=K, **kw), host_only=True)


@pytest.mark.parametrize("align", [1, 64, 128, 4096])
@pytest.mark.parametrize("dt", [np.float64, np.float32, np.int32])
def test_offsets_match_reference_formula(align, dt):
    K = [5, 10, 8]
    r = host_runner(K)
    parts = [np.zeros(k * 7, dtype=dt) for k in K]
    r.DefineBindings(Input("U").Bind(parts).Align(align))
    r.AllocateDevice()
    off = r.GetOffsets("U")
    ref, _ = g.aligned_offsets(K, sum(K) * 7 * np.dtype(dt).itemsize, np.dtype(dt).itemsize, align)
    assert off == ref
    assert all(b >= a for a, b in zip(off, off[1:]))
    assert off[1] - off[0] >= K[0] * 7


def test_binding_errors():
    r = host_runner([5, 10, 8])
    with pytest.raises(d.DGKError, match="non-partitioned array"):
        r.DefineBindings(Input("A").Bind(np.zeros(23)))
    with pytest.raises(d.DGKError, match="partition count mismatch"):
        r.DefineBindings(Input("B").Bind([np.zeros(5), np.zeros(10)]))
    r1 = host_runner([10])
    with pytest.raises(d.DGKError, match="partitioned data"):
        r1.DefineBindings(Input("C").Bind([np.zeros(5)]))
    r.DefineBindings(Input("ok").Bind([np.zeros(5), np.zeros(10), np.zeros(8)]), Temp("t").Size(23))
    r.AllocateDevice()
    with pytest.raises(d.DGKError, match="after AllocateDevice"):
        r.DefineBindings(Input("late").Bind([np.zeros(5), np.zeros(10), np.zeros(8)]))
    with pytest.raises(d.DGKError, match="already allocated"):
        r.AllocateDevice()
    with pytest.raises(d.DGKError, match="no binding"):
        r.ConfigureKernel("k", r.Param("missing"))
    with pytest.raises(d.DGKError, match="not configured"):
        r.ExecuteKernel("never")
    r.ConfigureKernel("k", r.Param("ok"))
    with pytest.raises(d.DGKError) as ei:
        r.BuildKernel("differentiate", "k")
    assert ei.value.code == _lib.ERR_NO_DEVICE


def test_runner_create_errors():
    with pytest.raises(d.DGKError, match="KpartMax exceeds"):
        host_runner([1 << 20 + 1])
    with pytest.raises(d.DGKError, match="empty"):
        host_runner([])


def test_configure_before_allocate():
    r = host_runner([4])
    r.DefineBindings(Input("A").Bind(np.zeros(4)))
    with pytest.raises(d.DGKError, match="not allocated"):
        r.ConfigureKernel("k", r.Param("A"))


def test_preamble_and_signature_text():
    r = host_runner([3, 4, 10])
    Dr = np.arange(9, dtype=float).reshape(3, 3)
    r.DefineBindings(
        Input("Dr").Bind(Dr).ToMatrix().Static(),
        Input("Mdev").Bind(np.eye(2)).ToMatrix(),
        Input("U").Bind([np.zeros(3 * 3), np.zeros(4 * 3), np.zeros(10 * 3)]),
        Output("V").Bind([np.zeros(3 * 3, dtype=np.float32), np.zeros(4 * 3, dtype=np.float32),
                          np.zeros(10 * 3, dtype=np.float32)]),
        Scalar("alpha").Bind(2.0),
    )
    r.AllocateDevice()
    pre = r.GeneratePreamble()
    assert "typedef long int_t;" in pre
    assert "#define NPART 3" in pre and "#define KpartMax 10" in pre
    assert "const double Dr[3][3] = {" in pre
    assert "{0.0000000000000000e+00, 3.0000000000000000e+00, 6.0000000000000000e+00}" in pre  # column-major
    assert "#define MATMUL_Dr(IN, OUT, K_VAL)" in pre and "#define MATMUL_ADD_Dr(IN, OUT, K_VAL)" in pre
    assert "sum += Dr[jj][ii] * (IN)[elem * 3 + jj];" in pre
    assert "sum += Mdev[jj * 2 + ii] * (IN)[elem * 2 + jj];" in pre
    assert "#define U_PART(part) ((double*)(U_global + U_offsets[part]))" in pre
    assert "#define V_PART(part) ((float*)(V_global + V_offsets[part]))" in pre
    r.ConfigureKernel("k", r.Param("U").CopyTo(), r.Param("Dr"), r.Param("V").CopyBack(), r.Param("Mdev"),
                      r.Param("alpha"))
    sig = r.GetKernelSignatureForConfig("k").split(",\n\t")
    assert sig == ["const int_t* K", "const double* Mdev", "const double* U_global", "const int_t* U_offsets",
                   "float* V_global", "const int_t* V_offsets", "double alpha"]
    r32 = host_runner([4], IntType=d.INT32)
    r32.DefineBindings(Input("A").Bind(np.zeros(4)))
    r32.AllocateDevice()
    assert "typedef int int_t;" in r32.GeneratePreamble()


def test_abi_exports_every_declared_symbol():
    with open(os.path.join(ROOT, "include", "dgk.h")) as f:
        decl = set(re.findall(r"^(?:int|const char \*)\s*(dgk_\w+)\(", f.read(), re.M))
    assert decl, "no declarations parsed"
    assert decl == set(_lib.SIGNATURES), "Python signatures out of sync with include/dgk.h"
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (dgk_\w+)", out))
    assert decl <= exported, f"missing exports: {sorted(decl - exported)}"
    L = ctypes.CDLL(_lib.LIB_PATH)
    for name in decl:
        assert getattr(L, name)


def test_create_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(d.DGKError) as ei:
        Runner(Config(K=[4]))
    assert ei.value.code == _lib.ERR_NO_DEVICE
