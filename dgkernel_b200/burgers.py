"""3-D scalar Burgers on a periodic Kuhn-cube mesh, assembled through the runner API.

This is the calling pattern of examples/3d_scalar_burgers_equation.go:168-471 with the full strong-form
right-hand side: bindings for state, geometry, face data and reference matrices; FP64 geometry and face
maps computed on the GPU; the FaceConnector exchange fused into a gather map; one `rhsStage` kernel per
LSERK4 stage.
"""
from __future__ import annotations

import math

import numpy as np

from . import mesh as M
from .element import Element
from .runner import (Config, Float32, Float64, INT32, INT64, Runner, Scalar, Temp, Input, WarpAlign)
from ._lib import check, lib


def mlp_param_count(nin: int) -> int:
    n = C.c_int64()
    check(lib().dgk_mlp_param_count(int(nin), C.byref(n)))
    return n.value

import ctypes as C

# Carpenter-Kennedy five-stage LSERK4 (examples/3d_scalar_burgers_equation.go:138-151)
RK4A = (0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
        -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0)
RK4B = (1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
        1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
        2277821191437.0 / 14882151754819.0)

DEFAULT_SEED = 20261203
GEO = ("Rx", "Ry", "Rz", "Sx", "Sy", "Sz", "Tx", "Ty", "Tz")
FACE = ("nx", "ny", "nz", "Fscale")
DERIV = ("DuDx", "DuDy", "DuDz")


class UniformStream:
    """Sequential splitmix64 uniforms drawn in blocks from the library."""

    def __init__(self, seed: int, block: int = 4096):
        self.seed, self.block, self.buf, self.pos = seed, block, M.splitmix_uniform(seed, block), 0

    def uniform(self) -> float:
        if self.pos == len(self.buf):
            self.buf = M.splitmix_uniform(self.seed, len(self.buf) * 2)
        v = float(self.buf[self.pos])
        self.pos += 1
        return v

    def normal(self) -> float:
        u1 = 1.0 - self.uniform()
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def random_modes(seed: int, nmodes: int = 8, kmax: int = 3, sigma: float = 0.1) -> np.ndarray:
    """Rows (kx, ky, kz, a, phi): integer k in [-kmax,kmax]^3 with 0 < |k| <= kmax by rejection,
    a ~ N(0, sigma^2), phi ~ U[0, 2 pi)."""
    rng = UniformStream(seed)
    rows = []
    for _ in range(nmodes):
        while True:
            k = [int(math.floor(rng.uniform() * (2 * kmax + 1))) - kmax for _ in range(3)]
            k2 = sum(v * v for v in k)
            if 0 < k2 <= kmax * kmax:
                break
        a = sigma * rng.normal()
        phi = 2.0 * math.pi * rng.uniform()
        rows.append([k[0], k[1], k[2], a, phi])
    return np.array(rows, dtype=np.float64)


def bary_matrix(el) -> np.ndarray:
    """Np x 4 barycentric coordinates (vertices A=(-1,-1,-1), B=(1,-1,-1), C=(-1,1,-1), D=(-1,-1,1)) of the
    element's nodes; the mixed stage subtracts the linear interpolant through the vertex nodes with them."""
    r, s, t = el.r, el.s, el.t
    return np.stack((-(1 + r + s + t) / 2, (1 + r) / 2, (1 + s) / 2, (1 + t) / 2), axis=1)


MIXED = "mixed"


def ensemble_sizes(count: int = 256, lo: int = 6, hi: int = 24, seed: int = DEFAULT_SEED):
    """Cube counts per axis of a seeded batch of instances: n_i uniform on {lo..hi} from a splitmix64 stream."""
    u = M.splitmix_uniform(seed, count)
    return [lo + int(math.floor(v * (hi - lo + 1))) for v in u]


def _concat_meshes(sizes):
    """Independent periodic n^3 x 6 Kuhn meshes side by side: vertex and element ids offset per instance,
    EToP = instance index, so every instance is one partition with no face shared with another."""
    VX, VY, VZ, EToV, EToE, EToF, EToP = [], [], [], [], [], [], []
    voff = eoff = 0
    for i, n in enumerate(sizes):
        vx, vy, vz, etov, etovp, _ = M.kuhn_mesh(int(n), 1)
        etoe, etof = M.ti_connect3d(etovp)
        VX.append(vx), VY.append(vy), VZ.append(vz)
        EToV.append(etov + voff)
        EToE.append(etoe + eoff)
        EToF.append(etof)
        EToP.append(np.full(etov.shape[0], i, dtype=np.int64))
        voff += len(vx)
        eoff += etov.shape[0]
    cat = lambda xs: np.ascontiguousarray(np.concatenate(xs))
    return cat(VX), cat(VY), cat(VZ), cat(EToV), cat(EToE), cat(EToF), cat(EToP)


class _TetBurgers:
    """Assembly shared by the single-mesh problem and the batch of instances: bindings for state, geometry,
    face data and reference matrices; FP64 geometry, normals and periodic VmapP computed on the GPU; the
    FaceConnector exchange fused into a gather map; one stage operator.

    dtype float64 / float32: the plain stage (`rhsStage`) with state, metrics and face data in that type.
    dtype "mixed": the mixed-precision stage (`rhsStageMixed`): compensated FP32 state uhi + ulo, FP32
    residual, compact affine geometry derived from the FP64 metrics; `get("u")` joins the pair in FP64."""

    def _assemble(self, N, VX, VY, VZ, EToV, EToE, EToF, EToP, Kpart, dtype, stream, viscosity=None):
        self.N = N
        self.visc = viscosity
        self.mixed = isinstance(dtype, str) and dtype == MIXED
        self.dtype = np.dtype(np.float64) if self.mixed else np.dtype(dtype)
        dt_code = Float64 if self.dtype == np.float64 else Float32
        el = self.el = Element(N)
        Np, Nfp = el.Np, el.Nfp
        NF = 4 * Nfp
        self.EToV, self.EToP = EToV, EToP
        K = self.K = EToV.shape[0]
        self.Kpart = list(Kpart)
        r = self.runner = Runner(Config(K=self.Kpart), stream=stream)
        sn = el.ShortName
        state = ("u", "X", "Y", "Z") if self.mixed else ("u", "uNext", "resu", "X", "Y", "Z")
        params = [Temp(nm).Type(dt_code).Size(K * Np) for nm in state + GEO]
        params += [Temp(nm).Type(dt_code).Size(K * NF) for nm in FACE]
        params += [Temp("gmap").Type(INT32).Size(K * NF), Temp("vmapP").Type(INT64).Size(K * NF)]
        if getattr(self, "derivatives", False):
            # outputs of the standalone volume-derivative operator (`differentiate`) on this mesh
            params += [Temp(nm).Type(dt_code).Size(K * Np) for nm in DERIV]
        if self.mixed:
            # 128-byte partition starts: the mixed stage streams each partition's slots with 16-byte bulk copies
            params += [Temp(nm).Type(Float32).Size(K * Np).Align(WarpAlign)
                       for nm in ("uhi", "ulo", "uhiNext", "uloNext", "resu")]
            params += [Input(f"Bary_{sn}").Bind(bary_matrix(el)).ToMatrix().Static()]
        if getattr(self, "learned", None):
            if not self.mixed:
                raise ValueError("the learned-sensor viscosity runs on the mixed stage (dtype MIXED, mma=True)")
            params += [Input(f"Vinv_{sn}").Bind(el.Vinv).ToMatrix().Static()]
            params += [Input("MLP").Bind(np.zeros((1, mlp_param_count(Np)))).ToMatrix().DeviceMemType(Float32)]
        if self.visc:
            if self.mixed or self.dtype != np.float64:
                raise ValueError("the artificial-viscosity stage runs in float64")
            params += [Temp(nm).Type(Float64).Size(K * Np) for nm in ("eps", "qx", "qy", "qz")]
            params += [Temp("feat").Type(Float32).Size(K * Np), Temp("sigma").Type(Float32).Size(K),
                       Temp("mlpSigma").Type(Float32).Size(K)]
            params += [Input(f"Vinv_{sn}").Bind(el.Vinv).ToMatrix().Static()]
            params += [Input("MLP").Bind(np.zeros((1, mlp_param_count(Np)))).ToMatrix().DeviceMemType(Float32)]
        params += [Input(f"{m}_{sn}").Bind(getattr(el, m)).ToMatrix().Static() for m in ("Dr", "Ds", "Dt", "LIFT")]
        params += [Input("Fmask").Bind(el.Fmask.astype(np.float64)).ToMatrix().DeviceMemType(INT32)]
        params += [Scalar("a").Type(Float64), Scalar("b").Type(Float64), Scalar("dt").Type(Float64)]
        r.DefineBindings(*params)
        r.AllocateDevice()
        # FP64 geometry, normals and periodic VmapP on the GPU
        names = ["X", "Y", "Z", *GEO, None, "nx", "ny", "nz", None, "Fscale", None, "vmapP"]
        carr = (C.c_char_p * 20)(*[None if v is None else v.encode() for v in names])
        hmin = C.c_double()
        check(lib().dgk_setup_geometry(r._h, el._h, len(VX), _pd(VX), _pd(VY), _pd(VZ), _pi(EToV), _pi(EToE),
                                       _pi(EToF), getattr(self, "period", 2.0), carr, C.byref(hmin)), r._h)
        self.hmin = hmin.value
        # FaceConnector pick/place fused into one gather map over the state array's partition offsets
        self.vmapP = np.zeros(K * NF, dtype=np.int64)
        r.CopyFromDevice("vmapP", self.vmapP)
        self.node_off = r.GetOffsets("uhi" if self.mixed else "u")
        self.gmap = M.face_gather_map(K, 4, Nfp, Np, self.vmapP, EToP, self.node_off)
        r.CopyToDevice("gmap", self.gmap)

    def _finish(self, cfl, conservative, warps=None, ring=None, eps0=1.0, c0=0.0, kappa=1.0, conf=(0.1, 0.9)):
        r, el = self.runner, self.el
        sn = el.ShortName
        fixed_m = [f"Dr_{sn}", f"Ds_{sn}", f"Dt_{sn}", f"LIFT_{sn}", "Fmask"]
        if self.mixed:
            r.ConfigureKernel("splitState", r.Param("u"), r.Param("uhi"), r.Param("ulo"))
            r.BuildKernel("splitState", "splitState")
            r.ConfigureKernel("joinState", r.Param("u"), r.Param("uhi"), r.Param("ulo"))
            r.BuildKernel("joinState", "joinState")
            r.ExecuteKernel("splitState")
            fixed = ["uhi", "ulo", "uhiNext", "uloNext", "resu", *GEO, *FACE, "gmap", *fixed_m, f"Bary_{sn}"]
        else:
            fixed = ["u", "uNext", "resu", *GEO, *FACE, "gmap", *fixed_m]
        self.conservative = conservative
        self.u0 = self.get("u")
        self.dt = cfl * self.hmin / float(np.max(np.abs(self.u0)))
        if self.visc or getattr(self, "learned", None):
            self.av = {"eps0": eps0, "c0": c0, "kappa": kappa, "lo": conf[0], "hi": conf[1]}
            fs = self.get("Fscale").reshape(self.K, -1)
            self.eps_max = eps0 * float(np.max(2.0 / fs.max(axis=1))) / self.N
            if self.eps_max > 0:  # diffusive limit of the explicit step
                self.dt = min(self.dt, cfl * self.hmin ** 2 / self.eps_max)
        if getattr(self, "learned", None):
            fixed += [f"Vinv_{self.el.ShortName}", "MLP"]
        if self.visc:
            sn = self.el.ShortName
            fixed += ["eps", "qx", "qy", "qz", f"Vinv_{sn}", "MLP"]
            feats = ["u", *GEO, *FACE, "gmap", *fixed_m, f"Vinv_{sn}", "MLP", "feat", "sigma", "mlpSigma"]
            r.ConfigureKernel("sensorFeatures", *[r.Param(p) for p in feats])
        r.ConfigureKernel("rhsStage", *[r.Param(p) for p in fixed], r.Param("a"), r.Param("b"), r.Param("dt"))
        self.stage = 0
        self.build_stage(warps=warps, ring=ring)

    def _av_args(self, sensor):
        a = self.av
        return (f"sensor={sensor},eps0={a['eps0']!r},c0={a['c0']!r},kappa={a['kappa']!r},"
                f"lo={a['lo']!r},hi={a['hi']!r}")

    def op_id(self, warps=None, ring=None) -> str:
        """Operator id of the stage kernel, with the launch shape (mixed stage) when given."""
        if self.visc:
            return f"rhsStageAV({self._av_args(self.visc)})"
        if not self.mixed:
            if getattr(self, "compact", False):
                return f"rhsStage(conservative={self.conservative},compact=1)"
            return f"rhsStage(conservative={self.conservative})"
        args = [f"conservative={self.conservative}"]
        if getattr(self, "tensor", None) is not None:
            args.append(f"tensor={int(self.tensor)}")
        if getattr(self, "mma", None):
            args.append("mma=1")
        if getattr(self, "learned", None):
            args.append(self._av_args(self.learned))
        if warps:
            args.append(f"warps={warps}")
        if ring:
            args.append(f"ring={ring}")
        return "rhsStageMixed(" + ",".join(args) + ")"

    def build_stage(self, warps=None, ring=None, mma=None):
        """(Re)build the stage operator, optionally with a given launch shape (and, for the mixed stage, the
        product path: mma=True puts the element-local products on the tensor cores)."""
        if mma is not None:
            self.mma = bool(mma)
        self.shape = {"warps": warps, "ring": ring, "mma": bool(getattr(self, "mma", None))}
        self.runner.BuildKernel(self.op_id(warps, ring), "rhsStage")

    def set_sensor(self, sensor: str, params=None):
        """Viscosity stage (or the learned-sensor mixed stage): switch the sensor ("none", "pp", "mlp"; "mlp0" on
        the mixed stage; for the network sensors its float32 parameters) and rebuild the stage."""
        if not (self.visc or getattr(self, "learned", None)):
            raise ValueError("problem built without viscosity")
        if params is not None:
            self.runner.CopyToDevice("MLP", np.asarray(params, dtype=np.float64).reshape(1, -1))
        if self.visc:
            self.visc = sensor
        else:
            self.learned = sensor
        self.build_stage()

    def sensor_features(self, sensor: str = "pp"):
        """(unit-norm modal coefficients [K, Np], PP activation [K], network output [K] or None) of the current
        state, from the stage's own sensor pass."""
        r = self.runner
        r.BuildKernel(f"sensorFeatures({self._av_args(sensor)})", "sensorFeatures")
        r.ExecuteKernel("sensorFeatures")
        feat = np.zeros(self.K * self.el.Np, dtype=np.float32)
        sig = np.zeros(self.K, dtype=np.float32)
        r.CopyFromDevice("feat", feat)
        r.CopyFromDevice("sigma", sig)
        mo = None
        if sensor == "mlp":
            mo = np.zeros(self.K, dtype=np.float32)
            r.CopyFromDevice("mlpSigma", mo)
        return feat.reshape(self.K, self.el.Np), sig, mo

    @property
    def dofs(self) -> int:
        return self.K * self.el.Np

    def get(self, name: str) -> np.ndarray:
        if self.mixed and name == "u":
            self.runner.ExecuteKernel("joinState")
        n = self.K * (self.el.Np if name not in FACE + ("gmap", "vmapP") else 4 * self.el.Nfp)
        dt = {"gmap": np.int32, "vmapP": np.int64}.get(name, self.dtype)
        if self.mixed and name in ("uhi", "ulo", "resu", "uhiNext", "uloNext"):
            dt = np.float32
        out = np.zeros(n, dtype=dt)
        self.runner.CopyFromDevice(name, out)
        return out

    def set(self, name: str, host: np.ndarray):
        self.runner.CopyToDevice(name, np.ascontiguousarray(host))
        if self.mixed and name == "u":
            self.runner.ExecuteKernel("splitState")

    def differentiate(self, repeats: int = 1):
        """DuDx, DuDy, DuDz of the current u through the `differentiate` operator (Dr/Ds/Dt then the nine
        per-node metrics; tetnudg/tet_nudg_mesh_physical_derivative_test.go:921-1078), `repeats` launches."""
        if not getattr(self, "derivatives", False) or self.mixed:
            raise ValueError("problem built without derivative outputs (derivatives=True, float dtype)")
        r, sn = self.runner, self.el.ShortName
        if "differentiate" not in r.KernelConfigs:
            r.ConfigureKernel("differentiate", r.Param("u"), *[r.Param(n) for n in GEO],
                              *[r.Param(n) for n in DERIV], *[r.Param(f"{m}_{sn}") for m in ("Dr", "Ds", "Dt")])
            r.BuildKernel("differentiate", "differentiate")
        for _ in range(repeats):
            r.ExecuteKernel("differentiate")

    def run_stages(self, nstages: int):
        """Advance by nstages LSERK4 stages (stage index continues across calls)."""
        for _ in range(nstages):
            s = self.stage % 5
            self.runner.ExecuteKernel("rhsStage", RK4A[s], RK4B[s], self.dt)
            self.stage += 1

    def capture_steps(self, nsteps: int = 2):
        """CUDA graph of `nsteps` whole LSERK4 steps (5 stages each; nsteps even so that the ping-pong state
        returns to its buffers); replay with `run_graph`.  Must start at a step boundary."""
        if self.stage % 5 or nsteps < 2 or nsteps % 2:
            raise ValueError("capture whole steps, an even number of them, from a step boundary")
        rows = [(RK4A[s % 5], RK4B[s % 5], self.dt) for s in range(5 * nsteps)]
        g = self.runner.CaptureGraph("rhsStage", rows)
        g.steps = nsteps
        return g

    def run_graph(self, graph, repeats: int = 1):
        graph.Launch(repeats)
        self.stage += 5 * graph.steps * repeats

    def free(self):
        self.runner.Free()


class BurgersProblem(_TetBurgers):
    """Device-resident Burgers problem of order N on one periodic n^3 x 6 Kuhn mesh with nslab x-slab
    partitions (u0: "sine", "shock", "smooth" or "modes"; dtype float64, float32 or "mixed")."""

    def __init__(self, N: int, n: int, nslab: int = 1, dtype=np.float64, u0: str = "sine", seed: int = DEFAULT_SEED,
                 cfl: float = 0.3, conservative: int = 0, stream=None, u0_host=None, warps=None, ring=None,
                 viscosity=None, eps0: float = 1.0, c0: float = 0.0, kappa: float = 1.0, conf=(0.1, 0.9),
                 mode_sigma: float = 0.1, tensor=None, mma=None, derivatives=False, learned=None, compact=False):
        self.n, self.nslab = n, nslab
        # float64 stage on the compact layout: per-element geometry and compact connectivity (straight-sided
        # elements), the same FP64 tensor-path arithmetic as the plain stage
        self.compact = compact
        # mixed tensor-core stage with learned-sensor (or PP) artificial viscosity: "pp", "mlp" or "mlp0"
        self.learned = learned
        self.derivatives = derivatives  # also bind DuDx, DuDy, DuDz for the `differentiate` operator
        self.tensor = tensor  # mixed form: None = by order (tensor cores for orders 6, 7), True / False to force
        self.mma = mma  # mixed form, orders 1..4: element-local products on the tensor cores (3-part BF16)
        VX, VY, VZ, EToV, EToVp, EToP = M.kuhn_mesh(n, nslab)
        EToE, EToF = M.ti_connect3d(EToVp)
        K = EToV.shape[0]
        self._assemble(N, VX, VY, VZ, EToV, EToE, EToF, EToP, [K // nslab] * nslab, dtype, stream, viscosity)
        r = self.runner
        if u0_host is not None:
            r.CopyToDevice("u", np.ascontiguousarray(u0_host, dtype=self.dtype).reshape(-1))
        else:
            kinds = {"sine": (0, 0.0, 0.5), "shock": (0, 0.5, 1.0), "smooth": (1, 0.5, 0.25), "modes": (2, 0.5, 0.0)}
            kind, mean, amp = kinds[u0]
            modes = random_modes(seed, sigma=mode_sigma) if kind == 2 else np.zeros((0, 5))
            check(lib().dgk_init_field(r._h, b"u", b"X", b"Y", b"Z", kind, mean, amp, len(modes), _pd(modes)), r._h)
        self._finish(cfl, conservative, warps, ring, eps0, c0, kappa, conf)


def partition_order(EToP):
    """Element order that makes every partition a contiguous block (ascending partition id, then ascending
    element id: the FaceConnector's local numbering, utils/face_connector.go:93-118), the partition ids in
    that order, and the element count of each."""
    EToP = np.asarray(EToP, dtype=np.int64)
    if EToP.size and EToP.min() < 0:
        raise ValueError("every element needs a partition (EToP has unassigned elements)")
    order = np.argsort(EToP, kind="stable")
    ids, counts = np.unique(EToP, return_counts=True)
    return order, ids, [int(c) for c in counts]


class BurgersMesh(_TetBurgers):
    """Burgers problem of order N on an unstructured tetrahedral mesh (vertices VX, VY, VZ, EToV [K, 4], optional
    EToP, e.g. from mesh.read_gambit), not periodic: faces without a neighbour keep VmapP = VmapM
    (element/library/gonudg/buildmaps3d.go:34, 156-173), so their Lax-Friedrichs difference vanishes.  Elements
    are stored partition by partition (partition_order); `order` maps stored position -> input element."""

    def __init__(self, N: int, VX, VY, VZ, EToV, EToP=None, dtype=np.float64, u0: str = "sine", cfl: float = 0.3,
                 conservative: int = 0, stream=None, mma=None, tensor=None):
        EToV = np.ascontiguousarray(EToV, dtype=np.int64)
        K = EToV.shape[0]
        EToP = np.zeros(K, dtype=np.int64) if EToP is None else np.asarray(EToP, dtype=np.int64)
        order, self.part_ids, Kpart = partition_order(EToP)
        EToV = np.ascontiguousarray(EToV[order])
        EToPc = np.ascontiguousarray(np.repeat(np.arange(len(Kpart), dtype=np.int64), Kpart))
        EToE, EToF = M.ti_connect3d(EToV)
        self.order, self.period, self.mma, self.tensor = order, 0.0, mma, tensor
        VX, VY, VZ = (np.ascontiguousarray(v, dtype=np.float64) for v in (VX, VY, VZ))
        self._assemble(N, VX, VY, VZ, EToV, EToE, EToF, EToPc, Kpart, dtype, stream)
        kinds = {"sine": (0, 0.0, 0.5), "shock": (0, 0.5, 1.0), "smooth": (1, 0.5, 0.25)}
        kind, mean, amp = kinds[u0]
        r = self.runner
        check(lib().dgk_init_field(r._h, b"u", b"X", b"Y", b"Z", kind, mean, amp, 0, _pd(np.zeros(5))), r._h)
        self._finish(cfl, conservative)


class BurgersEnsemble(_TetBurgers):
    """A batch of independent Burgers instances of order N, instance i on its own periodic n_i^3 x 6 Kuhn mesh
    (uneven K_i = 6 n_i^3), all in one runner with one partition per instance, so that one stage launch (and
    one persistent grid) advances every instance.  Instance i starts from 0.5 + 8 random modes drawn with
    seed + i; all instances share one time step, the CFL step of the most restrictive one."""

    def __init__(self, N: int, sizes, dtype=MIXED, seed: int = DEFAULT_SEED, cfl: float = 0.3, conservative: int = 0,
                 stream=None, warps=None, ring=None, mma=None):
        self.sizes = [int(n) for n in sizes]
        self.mma = mma
        VX, VY, VZ, EToV, EToE, EToF, EToP = _concat_meshes(self.sizes)
        Kpart = [6 * n ** 3 for n in self.sizes]
        self._assemble(N, VX, VY, VZ, EToV, EToE, EToF, EToP, Kpart, dtype, stream)
        r = self.runner
        modes = np.ascontiguousarray(np.concatenate([random_modes(seed + i) for i in range(len(self.sizes))]))
        check(lib().dgk_init_field_parts(r._h, b"u", b"X", b"Y", b"Z", 0.5, 8, _pd(modes)), r._h)
        self.modes = modes.reshape(len(self.sizes), 8, 5)
        self._finish(cfl, conservative, warps, ring)

    def instance(self, i: int, u: np.ndarray = None) -> np.ndarray:
        """Instance i's nodal values (FP64, element-contiguous) from a packed state (default: the current one)."""
        u = self.get("u") if u is None else u
        off = int(sum(self.Kpart[:i])) * self.el.Np
        return u[off:off + self.Kpart[i] * self.el.Np]


def _pd(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _pi(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))
