"""Python mirror of DGKernel's Go `runner` API over libdgk.so.

Names, argument meaning and error behaviour follow the reference (runner/runner.go, runner/binding.go,
runner/kernel_config.go, runner/kernel_execution.go, runner/builder/builder_param.go), so that code and tests
written against the runner read the same here.  Host data follows the Go binding kinds:

  * 1-D numpy array            -> []T (flat, element-contiguous)
  * 2-D numpy array            -> mat.Matrix (row-major; copies transpose to column-major)
  * list of 1-D / 2-D arrays   -> [][]T / []mat.Matrix (one entry per partition)
  * Python or numpy scalar     -> scalar

BuildKernel(source, name) selects a precompiled sm_100a operator: `source` is an operator id such as
"differentiate" or "rhsStage(uNext=u2)" (OKL source text is not compiled).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, List, Optional

import numpy as np

from ._lib import DGKError, check, lib

# builder.DataType (runner/builder/builder.go:12-20)
Float32, Float64, INT32, INT64 = 1, 2, 3, 4
# builder.AlignmentType (runner/builder/builder.go:24-30)
NoAlignment, CacheLineAlign, WarpAlign, PageAlign = 1, 64, 128, 4096
# builder.Direction (runner/builder/builder_param.go:10-17)
DirectionInput, DirectionOutput, DirectionInOut, DirectionTemp, DirectionScalar = range(5)
# ActionFlags (runner/binding.go:15-26)
NoAction, CopyTo, CopyBack = 0, 2, 4
Copy = CopyTo | CopyBack

_NP2DT = {np.dtype(np.float32): Float32, np.dtype(np.float64): Float64, np.dtype(np.int32): INT32,
          np.dtype(np.int64): INT64}
_DT2NP = {v: k for k, v in _NP2DT.items()}


def dtype_of(a) -> int:
    dt = np.asarray(a).dtype
    if dt not in _NP2DT:
        raise TypeError(f"unsupported host dtype {dt}")
    return _NP2DT[dt]


@dataclass
class Config:
    """builder.Config (runner/builder/builder.go:66-69)."""
    K: List[int]
    IntType: int = 0


@dataclass
class ParamSpec:
    Name: str
    Direction: int
    HostBinding: Any = None
    DataType: int = 0
    Size: int = 0
    DoCopyTo: bool = False
    DoCopyBack: bool = False
    ConvertType: int = 0
    Alignment: int = 0
    IsMatrix: bool = False
    IsStatic: bool = False
    IsPartitioned: bool = False
    PartitionCount: int = 0


class ParamBuilder:
    """Fluent parameter builder (runner/builder/builder_param.go:56-196)."""

    def __init__(self, name: str, direction: int):
        self.Spec = ParamSpec(name, direction)

    def Bind(self, host) -> "ParamBuilder":
        s = self.Spec
        s.HostBinding = host
        if isinstance(host, (list, tuple)):
            s.IsPartitioned, s.PartitionCount = True, len(host)
            s.Size = int(sum(np.asarray(h).size for h in host))
            s.DataType = dtype_of(host[0]) if host else 0
        elif isinstance(host, np.ndarray):
            s.Size = int(host.size)
            s.DataType = dtype_of(host)
        else:
            s.Size = 1
            s.DataType = INT64 if isinstance(host, (int, np.integer)) and not isinstance(host, bool) else Float64
            if isinstance(host, np.floating):
                s.DataType = dtype_of(np.asarray(host))
        return self

    def Copy(self):
        self.Spec.DoCopyTo = self.Spec.DoCopyBack = True
        return self

    def CopyTo(self):
        self.Spec.DoCopyTo = True
        return self

    def CopyBack(self):
        self.Spec.DoCopyBack = True
        return self

    def NoCopy(self):
        self.Spec.DoCopyTo = self.Spec.DoCopyBack = False
        return self

    def DeviceMemType(self, t: int):
        self.Spec.ConvertType = t
        return self

    def Type(self, t: int):
        self.Spec.DataType = t
        return self

    def Size(self, n: int):
        self.Spec.Size = int(n)
        return self

    def ToMatrix(self):
        self.Spec.IsMatrix = True
        return self

    def Static(self):
        self.Spec.IsStatic = True
        return self

    def Align(self, a: int):
        self.Spec.Alignment = a
        return self

    def effective_type(self) -> int:
        return self.Spec.ConvertType or self.Spec.DataType


def Input(name):
    return ParamBuilder(name, DirectionInput)


def Output(name):
    return ParamBuilder(name, DirectionOutput)


def InOut(name):
    return ParamBuilder(name, DirectionInOut)


def Scalar(name):
    return ParamBuilder(name, DirectionScalar)


def Temp(name):
    return ParamBuilder(name, DirectionTemp)


class ParamConfig:
    """Per-kernel copy actions of a binding (runner/kernel_config.go:151-181)."""

    def __init__(self, name: str, known: bool):
        self.name, self.known, self.actions = name, known, NoAction

    def CopyTo(self):
        self.actions |= CopyTo
        return self

    def CopyBack(self):
        self.actions |= CopyBack
        return self

    def Copy(self):
        self.actions |= Copy
        return self

    def NoCopy(self):
        self.actions = NoAction
        return self


@dataclass
class _Binding:
    spec: ParamSpec
    host: Any
    host_dtype: int
    dev_dtype: int
    is_scalar: bool = False
    is_matrix: bool = False
    partitioned: bool = False
    layout: int = 0


@dataclass
class _Kernel:
    params: List[ParamConfig] = field(default_factory=list)
    built: bool = False


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class Runner:
    """runner.Runner over libdgk.so: NewRunner(device, Config) is Runner(Config)."""

    def __init__(self, config: Config, host_only: bool = False, stream: Optional[int] = None):
        L = lib()
        K = np.ascontiguousarray(np.asarray(config.K, dtype=np.int64))
        h = C.c_void_p()
        create = L.dgk_runner_create_host_only if host_only else L.dgk_runner_create
        check(create(K.ctypes.data_as(C.POINTER(C.c_int64)), len(K), int(config.IntType), C.byref(h)))
        self._h = h
        self.K = [int(k) for k in config.K]
        self.NumPartitions = len(self.K)
        self.KpartMax = max(self.K)
        self.IsPartitioned = self.NumPartitions > 1
        self.IsAllocated = False
        self.Bindings: dict = {}
        self.KernelConfigs: dict = {}
        if stream is not None:
            self.SetStream(stream)

    # -- lifecycle --------------------------------------------------------------------------------
    def Free(self):
        if getattr(self, "_h", None):
            lib().dgk_runner_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Free()
        except Exception:
            pass

    def _check(self, rc):
        check(rc, self._h)

    def SetStream(self, stream_handle: int):
        self._check(lib().dgk_set_stream(self._h, C.c_void_p(stream_handle)))

    def Sync(self):
        """Device.Finish (runner/kernel_execution.go:62)."""
        self._check(lib().dgk_sync(self._h))

    # -- bindings ---------------------------------------------------------------------------------
    def DefineBindings(self, *params: ParamBuilder):
        """DefineBindings (runner/binding.go:100-124)."""
        L = lib()
        for p in params:
            s = p.Spec
            if s.IsPartitioned and s.IsMatrix and s.IsStatic:
                raise DGKError(1, "static matrices cannot be partitioned")
            name = s.Name.encode()
            if s.Direction == DirectionScalar:
                v = None if s.HostBinding is None else C.byref(C.c_double(float(s.HostBinding)))
                self._check(L.dgk_bind_scalar(self._h, name, s.DataType or Float64, v))
                self.Bindings[s.Name] = _Binding(s, s.HostBinding, s.DataType, s.DataType, is_scalar=True)
                continue
            if s.IsMatrix and not s.IsPartitioned:
                m = np.ascontiguousarray(np.asarray(s.HostBinding, dtype=np.float64))
                if m.ndim != 2:
                    raise DGKError(1, f"matrix {s.Name} must be 2-D")
                self._check(L.dgk_bind_matrix(self._h, name, m.shape[0], m.shape[1],
                                              m.ctypes.data_as(C.POINTER(C.c_double)), int(s.IsStatic),
                                              p.effective_type() if s.ConvertType else Float64))
                self.Bindings[s.Name] = _Binding(s, m, Float64, s.ConvertType or Float64, is_matrix=True)
                continue
            host = s.HostBinding
            layout, rows, cols = 0, 0, 0
            part_vals = None
            if s.Direction == DirectionTemp:
                hdt = ddt = s.DataType or Float64
                total = s.Size
            elif host is None:
                hdt = ddt = p.effective_type() or Float64
                total = s.Size
            else:
                hdt = s.DataType
                ddt = s.ConvertType or hdt
                if isinstance(host, (list, tuple)):
                    part_vals = np.array([np.asarray(h).size for h in host], dtype=np.int64)
                    total = int(part_vals.sum())
                    first = np.asarray(host[0])
                    if first.ndim == 2:
                        layout, rows, cols = 1, first.shape[0], first.shape[1]
                else:
                    a = np.asarray(host)
                    total = a.size
                    if a.ndim == 2:
                        layout, rows, cols = 1, a.shape[0], a.shape[1]
            pc = 0 if part_vals is None else len(part_vals)
            pv = None if part_vals is None else part_vals.ctypes.data_as(C.POINTER(C.c_int64))
            self._check(L.dgk_bind_array(self._h, name, s.Direction, hdt, ddt, int(total), pc, pv, int(s.Alignment),
                                         layout, rows, cols))
            self.Bindings[s.Name] = _Binding(s, host, hdt, ddt, partitioned=pc > 0, layout=layout)

    def AllocateDevice(self):
        """AllocateDevice (runner/binding.go:339-384)."""
        self._check(lib().dgk_allocate(self._h))
        self.IsAllocated = True

    def GetOffsets(self, name: str) -> List[int]:
        out = np.zeros(self.NumPartitions + 1, dtype=np.int64)
        self._check(lib().dgk_get_offsets(self._h, name.encode(), out.ctypes.data_as(C.POINTER(C.c_int64))))
        return [int(v) for v in out]

    def DevicePtr(self, name: str) -> int:
        p = C.c_void_p()
        self._check(lib().dgk_device_ptr(self._h, name.encode(), C.byref(p)))
        return int(p.value or 0)

    # -- copies -----------------------------------------------------------------------------------
    def _host_view(self, b: _Binding, host):
        a = np.asarray(host)
        want = _DT2NP[b.host_dtype]
        if a.dtype != want or not a.flags.c_contiguous:
            raise DGKError(1, f"host buffer of {b.spec.Name} must be a C-contiguous {want} array")
        return a

    def _copy(self, name: str, to_device: bool, host=None):
        b = self.Bindings.get(name)
        if b is None:
            raise DGKError(3, f"binding {name} not found")
        if b.is_scalar:
            return
        host = b.host if host is None else host
        if host is None:
            return
        L = lib()
        if isinstance(host, (list, tuple)):
            for part, h in enumerate(host):
                a = self._host_view(b, h)
                fn = L.dgk_copy_partition_to_device if to_device else L.dgk_copy_partition_from_device
                self._check(fn(self._h, name.encode(), part, _ptr(a), a.nbytes))
            return
        a = self._host_view(b, host)
        fn = L.dgk_copy_to_device if to_device else L.dgk_copy_from_device
        self._check(fn(self._h, name.encode(), _ptr(a), a.nbytes))

    def CopyToDevice(self, name: str, host=None):
        """CopyToDevice (runner/memory_operations.go:219-229); `host` overrides the bound buffer."""
        self._copy(name, True, host)

    def CopyFromDevice(self, name: str, host=None):
        """CopyFromDevice (runner/memory_operations.go:231-241)."""
        self._copy(name, False, host)

    def CopyArrayToHost(self, name: str) -> np.ndarray:
        """All partitions of an array back to back, raw device order and type (runner/runner_copy.go:13-80).
        Each partition contributes K[part] x values-per-element values; the reference copies only K[part]
        values (runner/runner_copy.go:64-66)."""
        return np.concatenate([self.CopyPartitionToHost(name, p) for p in range(self.NumPartitions)])

    def CopyPartitionToHost(self, name: str, part: int) -> np.ndarray:
        """One partition in raw device order and type (runner/runner_copy.go:83-145)."""
        b = self.Bindings.get(name)
        if b is None or b.is_scalar:
            raise DGKError(3, f"array {name} not found")
        if part < 0 or part >= self.NumPartitions:
            raise DGKError(1, f"invalid partition ID: {part}")
        off = self.GetOffsets(name)
        total = sum(self.K)
        if b.partitioned:
            n = int(np.asarray(b.host[part]).size)
        else:
            n = (b.spec.Size // total) * self.K[part] if total else 0
        out = np.zeros(n, dtype=_DT2NP[b.dev_dtype])
        self._check(lib().dgk_copy_raw_from_device(self._h, name.encode(), off[part], _ptr(out), out.nbytes))
        return out

    # -- kernels ----------------------------------------------------------------------------------
    def Param(self, name: str) -> ParamConfig:
        return ParamConfig(name, name in self.Bindings)

    def ConfigureKernel(self, name: str, *params: ParamConfig):
        """ConfigureKernel (runner/kernel_config.go:51-91)."""
        if not self.IsAllocated:
            raise DGKError(2, "device memory not allocated - call AllocateDevice first")
        params = [p for p in params if p is not None]
        for p in params:
            if not p.known:
                raise DGKError(3, "parameter configuration has no binding")
        names = (C.c_char_p * len(params))(*[p.name.encode() for p in params])
        acts = (C.c_uint32 * len(params))(*[p.actions for p in params])
        self._check(lib().dgk_configure_kernel(self._h, name.encode(), len(params), names, acts))
        self.KernelConfigs[name] = _Kernel(list(params))
        return self.KernelConfigs[name]

    def GetKernelSignatureForConfig(self, name: str) -> str:
        """GetKernelSignatureForConfig (runner/kernel_execution.go:230-237)."""
        L = lib()
        n = L.dgk_kernel_signature(self._h, name.encode(), None, 0)
        if n <= 0:
            self._check(n if n else 1)
        buf = C.create_string_buffer(n + 1)
        self._check(L.dgk_kernel_signature(self._h, name.encode(), buf, n + 1))
        return buf.value.decode()

    def GeneratePreamble(self) -> str:
        """GeneratePreamble (runner/builder/builder.go:172-191)."""
        L = lib()
        n = L.dgk_generate_preamble(self._h, None, 0)
        buf = C.create_string_buffer(n + 1)
        self._check(L.dgk_generate_preamble(self._h, buf, n + 1))
        return buf.value.decode()

    def BuildKernel(self, kernel_source: str, kernel_name: str):
        """BuildKernel (runner/runner.go:88-126): `kernel_source` names a precompiled operator."""
        self._check(lib().dgk_build_kernel(self._h, kernel_name.encode(), kernel_source.encode()))
        if kernel_name in self.KernelConfigs:
            self.KernelConfigs[kernel_name].built = True

    def ExecuteKernel(self, name: str, *scalar_values):
        """ExecuteKernel (runner/kernel_execution.go:12-89): pre-copies, launch, post-copies."""
        if name not in self.KernelConfigs:
            raise DGKError(2, f"kernel {name} not configured - use ConfigureKernel first")
        kc = self.KernelConfigs[name]
        ptrs = (C.c_void_p * max(1, len(kc.params)))()
        keep, later = [], []
        for i, p in enumerate(kc.params):
            b = self.Bindings[p.name]
            if b.is_scalar or b.host is None or not (p.actions & Copy):
                continue
            if isinstance(b.host, (list, tuple)):  # partitioned: per-partition copies around the launch
                if p.actions & CopyTo:
                    self._copy(p.name, True)
                if p.actions & CopyBack:
                    later.append(p.name)
                continue
            a = self._host_view(b, b.host)
            keep.append(a)
            ptrs[i] = a.ctypes.data
        sv = np.ascontiguousarray(np.asarray(scalar_values, dtype=np.float64))
        self._check(lib().dgk_execute_kernel(self._h, name.encode(), len(sv), sv.ctypes.data_as(C.POINTER(C.c_double)),
                                             ptrs))
        for n in later:
            self._copy(n, False)

    def CaptureGraph(self, name: str, scalar_rows) -> Graph:
        """Record len(scalar_rows) (even) launches of kernel `name`, row l giving launch l's scalars, into one
        CUDA graph.  Nothing runs until Graph.Launch; ping-pong operators leave the bindings naming the newest
        state after every replay."""
        rows = np.ascontiguousarray(np.asarray(scalar_rows, dtype=np.float64).reshape(len(scalar_rows), -1))
        h = C.c_void_p()
        self._check(lib().dgk_capture_graph(self._h, name.encode(), rows.shape[0], rows.shape[1],
                                            rows.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h)))
        return Graph(self, h, rows.shape[0])


class Graph:
    """A captured sequence of launches of one built kernel (CUDA graph); Launch replays it on the runner's
    stream.  Free it before its runner."""

    def __init__(self, runner: "Runner", handle, nlaunch: int):
        self.runner, self._h, self.nlaunch = runner, handle, nlaunch

    def Launch(self, repeats: int = 1):
        self.runner._check(lib().dgk_graph_launch(self._h, int(repeats)))

    def Free(self):
        if getattr(self, "_h", None):
            lib().dgk_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Free()
        except Exception:
            pass


def NewRunner(config: Config, **kw) -> Runner:
    return Runner(config, **kw)
