"""Parity of the CUDA path (libdgk.so on a B200) with the CPU oracle, through the runner / C ABI.

Tolerances: FP64 results agree with the oracle to <= 1e-12 relative L2 (the oracle sums without FMA in the
OKL order; the GPU uses FMA and a different summation order).  FP32 state is compared with the FP64 oracle at
<= 2e-5 relative L2 after the stated number of stages.  Index maps are compared bit-exactly.
"""
import numpy as np
import pytest

import dgkernel_b200 as d
from dgkernel_b200 import mesh as M
from dgkernel_b200.burgers import BurgersProblem, RK4A, RK4B, GEO, FACE
from dgkernel_b200.runner import Config, Input, Output, InOut, Scalar, Temp, Runner, Float32, INT32, WarpAlign
from oracle import burgers_ref as b
from oracle import gonudg_ref as g
from oracle import oracle as O

from conftest import rel_l2

pytestmark = pytest.mark.gpu
FP64_TOL = 1e-12
FP32_TOL = 2e-5


@pytest.fixture(scope="module")
def c1():
    return b.Problem(2, 8, 4, "sine")


def split(a, K, per):
    out, o = [], 0
    for k in K:
        out.append(np.array(a[o:o + k * per], copy=True))  # copies: bound host buffers are written back
        o += k * per
    return out


def test_geometry_and_maps_match_oracle(c1):
    P = BurgersProblem(2, 8, 4, np.float64, "sine")
    assert np.array_equal(P.vmapP, c1.vmapP)
    assert abs(P.hmin - c1.hmin) < 1e-15 and abs(P.dt - c1.dt) < 1e-15
    assert rel_l2(P.get("X"), c1.X) < 1e-15
    for nm, ref in zip(GEO, (c1.geo.rx, c1.geo.ry, c1.geo.rz, c1.geo.sx, c1.geo.sy, c1.geo.sz, c1.geo.tx, c1.geo.ty,
                             c1.geo.tz)):
        assert rel_l2(P.get(nm), ref) < 1e-13, nm
    for nm, ref in zip(FACE, (c1.geo.nx, c1.geo.ny, c1.geo.nz, c1.geo.Fscale)):
        assert rel_l2(P.get(nm), ref) < 1e-13, nm
    assert rel_l2(P.u0, c1.u0) < 1e-15
    P.free()


@pytest.mark.parametrize("N", [2, 3, 4])
def test_differentiate_partitioned_aligned(N):
    ref = b.Problem(N, 4, 2, "sine")
    el = ref.el
    K = ref.Kpart
    Np = el.Np
    r = Runner(Config(K=K))
    # []mat.Matrix, Np x Kp row-major: copies transpose them to element-contiguous
    U = [np.ascontiguousarray(u.reshape(K[p], Np).T) for p, u in enumerate(split(ref.u0.reshape(-1), K, Np))]
    geo = [split(getattr(ref.geo, n).reshape(-1), K, Np) for n in ("rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz")]
    outs = [[np.zeros(k * Np) for k in K] for _ in range(3)]
    sn = f"NudgTet{N}"
    params = [Input(f"{m}_{sn}").Bind(getattr(el, m)).ToMatrix() for m in ("Dr", "Ds", "Dt")]
    params += [Input("U").Bind(U).Align(WarpAlign)]
    params += [Input(n).Bind(a).Align(WarpAlign) for n, a in zip(GEO, geo)]
    params += [Output(n).Bind(a).Align(WarpAlign) for n, a in zip(("DuDx", "DuDy", "DuDz"), outs)]
    r.DefineBindings(*params)
    r.AllocateDevice()
    r.ConfigureKernel("differentiate", r.Param("U").CopyTo(), *[r.Param(n).CopyTo() for n in GEO],
                      *[r.Param(n).CopyBack() for n in ("DuDx", "DuDy", "DuDz")],
                      *[r.Param(f"{m}_{sn}") for m in ("Dr", "Ds", "Dt")])
    r.BuildKernel("differentiate", "differentiate")
    r.ExecuteKernel("differentiate")
    want = O.differentiate(el, K, ref.u0, [getattr(ref.geo, n) for n in ("rx", "ry", "rz", "sx", "sy", "sz", "tx",
                                                                          "ty", "tz")])
    for got, w in zip(outs, want):
        assert rel_l2(np.concatenate(got), w) < FP64_TOL
    off = r.GetOffsets("U")
    assert off[1] % 16 == 0 and off[1] >= K[0] * Np  # 128-byte partition alignment in values
    r.Free()


def _rhs_runner(ref, dtype=np.float64, only=True, conservative=0):
    el = ref.el
    K, Np, NF = ref.Kpart, el.Np, 4 * el.Nfp
    dt_code = d.Float64 if dtype == np.float64 else Float32
    r = Runner(Config(K=K))
    sn = f"NudgTet{el.N}"
    params = [Temp(n).Type(dt_code).Size(ref.K * Np) for n in ("u", "rhs", "uNext", "resu") + GEO]
    params += [Temp(n).Type(dt_code).Size(ref.K * NF) for n in FACE]
    params += [Temp("gmap").Type(INT32).Size(ref.K * NF)]
    params += [Input(f"{m}_{sn}").Bind(getattr(el, m)).ToMatrix().Static() for m in ("Dr", "Ds", "Dt", "LIFT")]
    params += [Input("Fmask").Bind(el.Fmask.astype(float)).ToMatrix().DeviceMemType(INT32)]
    params += [Scalar("a"), Scalar("b"), Scalar("dt")]
    r.DefineBindings(*params)
    r.AllocateDevice()
    for n, a in zip(GEO + FACE, (ref.geo.rx, ref.geo.ry, ref.geo.rz, ref.geo.sx, ref.geo.sy, ref.geo.sz, ref.geo.tx,
                                 ref.geo.ty, ref.geo.tz, ref.geo.nx, ref.geo.ny, ref.geo.nz, ref.geo.Fscale)):
        r.CopyToDevice(n, np.ascontiguousarray(a.reshape(-1), dtype=dtype))
    gm = M.face_gather_map(ref.K, 4, el.Nfp, Np, ref.vmapP, ref.EToP, r.GetOffsets("u"))
    r.CopyToDevice("gmap", gm)
    mats = [r.Param(f"{m}_{sn}") for m in ("Dr", "Ds", "Dt", "LIFT")] + [r.Param("Fmask")]
    common = [r.Param(n) for n in GEO + FACE] + [r.Param("gmap")] + mats
    r.ConfigureKernel("rhs", r.Param("u"), r.Param("rhs"), *common)
    r.BuildKernel(f"rhsLF(conservative={conservative})", "rhs")
    r.ConfigureKernel("stage", r.Param("u"), r.Param("uNext"), r.Param("resu"), *common, r.Param("a"),
                      r.Param("b"), r.Param("dt"))
    r.BuildKernel(f"rhsStage(conservative={conservative})", "stage")
    return r


@pytest.mark.parametrize("N,n,slabs", [(1, 3, 3), (2, 4, 2), (3, 4, 4), (4, 3, 1), (5, 2, 2)])
@pytest.mark.parametrize("conservative", [0, 1])
def test_rhs_lf_matches_oracle(N, n, slabs, conservative):
    ref = b.Problem(N, n, slabs, "modes")
    r = _rhs_runner(ref, conservative=conservative)
    r.CopyToDevice("u", np.ascontiguousarray(ref.u0.reshape(-1)))
    r.ExecuteKernel("rhs")
    got = np.zeros(ref.K * ref.el.Np)
    r.CopyFromDevice("rhs", got)
    want = O.RunState(ref).rhs(ref.u0, conservative=conservative)
    assert rel_l2(got, want) < FP64_TOL
    r.Free()


def test_rhs_lf_fp32(c1):
    r = _rhs_runner(c1, np.float32)
    r.CopyToDevice("u", np.ascontiguousarray(c1.u0.reshape(-1), dtype=np.float32))
    r.ExecuteKernel("rhs")
    got = np.zeros(c1.K * c1.el.Np, dtype=np.float32)
    r.CopyFromDevice("rhs", got)
    assert rel_l2(got, O.RunState(c1).rhs(c1.u0)) < FP32_TOL
    r.Free()


def test_stage_trajectory_c1_fp64(c1):
    # 10 LSERK4 steps (50 stages, t = 0.75) of the order-2 8^3 x 6 sine case, before the unlimited solution blows up past the shock
    P = BurgersProblem(2, 8, 4, np.float64, "sine")
    u = np.ascontiguousarray(c1.u0.reshape(-1)).copy()
    resu = np.zeros_like(u)
    O.RunState(c1).run(u, resu, c1.dt, 50, threads=4)
    P.run_stages(50)
    assert rel_l2(P.get("u"), u) < FP64_TOL
    assert rel_l2(P.get("resu"), resu) < 1e-11
    P.free()


def test_stage_trajectory_fp32(c1):
    P = BurgersProblem(2, 8, 4, np.float32, "sine")
    u = np.ascontiguousarray(c1.u0.reshape(-1)).copy()
    resu = np.zeros_like(u)
    O.RunState(c1).run(u, resu, c1.dt, 25)
    P.run_stages(25)
    assert rel_l2(P.get("u"), u) < FP32_TOL
    P.free()


def test_reference_form_compute_rhs_and_update(c1):
    el, K, Np = c1.el, c1.Kpart, c1.el.Np
    sn = "NudgTet2"
    parts = lambda a: split(np.ascontiguousarray(a.reshape(-1)), K, Np)
    u, resu = parts(c1.u0), [np.full(k * Np, 0.25) for k in K]
    rhsu = [np.zeros(k * Np) for k in K]
    r = Runner(Config(K=K))
    params = [Input(f"{m}_{sn}").Bind(getattr(el, m)).ToMatrix().Static() for m in ("Dr", "Ds", "Dt")]
    params += [InOut("u").Bind(u), InOut("resu").Bind(resu), Output("rhsu").Bind(rhsu)]
    params += [Input(n).Bind(parts(getattr(c1.geo, n.lower()))) for n in GEO]
    params += [Scalar("rka").Bind(0.5), Scalar("rkb")]  # rka bound (used), rkb positional
    params += [Temp(t).Size(c1.K * Np) for t in ("ur", "us", "ut")]
    r.DefineBindings(*params)
    r.AllocateDevice()
    r.ConfigureKernel("computeRHS", r.Param("u").CopyTo(), r.Param("rhsu").CopyBack(),
                      *[r.Param(f"{m}_{sn}") for m in ("Dr", "Ds", "Dt")], *[r.Param(n).CopyTo() for n in GEO],
                      r.Param("ur"), r.Param("us"), r.Param("ut"))
    r.BuildKernel("computeRHS", "computeRHS")
    r.ConfigureKernel("updateSolution", r.Param("u").Copy(), r.Param("resu").Copy(), r.Param("rhsu"),
                      r.Param("rka"), r.Param("rkb"))
    r.BuildKernel("updateSolution", "updateSolution")
    r.ExecuteKernel("computeRHS")
    r.ExecuteKernel("updateSolution", 0.9, 0.01)  # 0.9 is shadowed by the bound rka = 0.5
    off = np.concatenate(([0], np.cumsum(np.array(K) * Np))).astype(np.int64)
    Karr = np.array(K, dtype=np.int64)
    uo = np.ascontiguousarray(c1.u0.reshape(-1)).copy()
    ro = np.full_like(uo, 0.25)
    rh = np.zeros_like(uo)
    tmp = [np.zeros_like(uo) for _ in range(3)]
    L = O.lib()
    L.ora_compute_rhs_volume(Np, O.cm(el.Dr), O.cm(el.Ds), O.cm(el.Dt), len(K), Karr, off, uo,
                             *[np.ascontiguousarray(getattr(c1.geo, n.lower()).reshape(-1)) for n in GEO], *tmp, rh, 1)
    assert rel_l2(np.concatenate(rhsu), rh) < FP64_TOL
    L.ora_update_ref(Np, len(K), Karr, off, uo, ro, rh, 0.5, 0.01)
    assert rel_l2(np.concatenate(u), uo) < FP64_TOL
    assert rel_l2(np.concatenate(resu), ro) < FP64_TOL
    r.Free()


def test_matmul_operator(c1):
    el, K, Np = c1.el, c1.Kpart, c1.el.Np
    U = split(np.ascontiguousarray(c1.u0.reshape(-1)), K, Np)
    out = [np.zeros(k * Np) for k in K]
    r = Runner(Config(K=K))
    r.DefineBindings(Input("Dr_NudgTet2").Bind(el.Dr).ToMatrix().Static(), Input("U").Bind(U),
                     Output("Ur").Bind(out))
    r.AllocateDevice()
    r.ConfigureKernel("mm", r.Param("U").CopyTo(), r.Param("Ur").CopyBack(), r.Param("Dr_NudgTet2"))
    r.BuildKernel("matmul(M=Dr_NudgTet2,IN=U,OUT=Ur)", "mm")
    r.ExecuteKernel("mm")
    off = np.concatenate(([0], np.cumsum(np.array(K) * Np))).astype(np.int64)
    want = np.zeros(c1.K * Np)
    O.lib().ora_matmul(O.cm(el.Dr), Np, Np, len(K), np.array(K, dtype=np.int64),
                       np.ascontiguousarray(c1.u0.reshape(-1)), off, want, off, 0)
    assert rel_l2(np.concatenate(out), want) < FP64_TOL
    r.Free()


def test_matmul_add_operator(c1):
    # MATMUL_ADD_<M> (runner/builder/builder.go:355-410): OUT += M x IN per element, OUT starting nonzero
    el, K, Np = c1.el, c1.Kpart, c1.el.Np
    U = split(np.ascontiguousarray(c1.u0.reshape(-1)), K, Np)
    start = np.random.default_rng(11).standard_normal(c1.K * Np)
    out = split(start.copy(), K, Np)
    r = Runner(Config(K=K))
    r.DefineBindings(Input("Ds_NudgTet2").Bind(el.Ds).ToMatrix().Static(), Input("U").Bind(U),
                     InOut("Us").Bind(out))
    r.AllocateDevice()
    r.ConfigureKernel("mma", r.Param("U").CopyTo(), r.Param("Us").Copy(), r.Param("Ds_NudgTet2"))
    r.BuildKernel("matmulAdd(M=Ds_NudgTet2,IN=U,OUT=Us)", "mma")
    r.ExecuteKernel("mma")
    off = np.concatenate(([0], np.cumsum(np.array(K) * Np))).astype(np.int64)
    want = start.copy()
    O.lib().ora_matmul(O.cm(el.Ds), Np, Np, len(K), np.array(K, dtype=np.int64),
                       np.ascontiguousarray(c1.u0.reshape(-1)), off, want, off, 1)
    assert rel_l2(np.concatenate(out), want) < FP64_TOL
    r.Free()


def test_copy_engine_conversions_and_transposes():
    K = [3, 5]
    rng = np.random.default_rng(7)
    a64 = [rng.standard_normal(k * 4) for k in K]
    i64 = [rng.integers(-1000, 1000, k * 4).astype(np.int64) for k in K]
    mats = [rng.standard_normal((4, k)) for k in K]  # []mat.Matrix 4 x Kp, row-major
    r = Runner(Config(K=K))
    r.DefineBindings(Input("A").Bind(a64).DeviceMemType(Float32), Input("I").Bind(i64).DeviceMemType(INT32),
                     InOut("Mt").Bind(mats).Align(128))
    r.AllocateDevice()
    for n in ("A", "I", "Mt"):
        r.CopyToDevice(n)
    got = [np.zeros(k * 4) for k in K]
    r.CopyFromDevice("A", got)
    for g_, a in zip(got, a64):
        assert np.array_equal(g_, a.astype(np.float32).astype(np.float64))
    goti = [np.zeros(k * 4, dtype=np.int64) for k in K]
    r.CopyFromDevice("I", goti)
    assert all(np.array_equal(x, y) for x, y in zip(goti, i64))
    # device holds each partition column-major (element-contiguous), like the reference's transposed copies
    for p in range(2):
        assert np.array_equal(r.CopyPartitionToHost("Mt", p), mats[p].T.reshape(-1))
    back = [np.zeros_like(m) for m in mats]
    r.CopyFromDevice("Mt", back)
    assert all(np.array_equal(x, y) for x, y in zip(back, mats))
    r.Free()


def test_bad_gather_index_is_reported_not_faulted(c1):
    r = _rhs_runner(c1)
    r.CopyToDevice("u", np.ascontiguousarray(c1.u0.reshape(-1)))
    gm = M.face_gather_map(c1.K, 4, c1.el.Nfp, c1.el.Np, c1.vmapP, c1.EToP, r.GetOffsets("u"))
    bad = gm.copy()
    bad[17] = 2 ** 30
    r.CopyToDevice("gmap", bad)
    r.ExecuteKernel("rhs")
    with pytest.raises(d.DGKError, match="gather index"):
        r.Sync()
    r.CopyToDevice("gmap", gm)  # the context stays usable
    r.ExecuteKernel("rhs")
    r.Sync()
    r.Free()


def test_full_size_conservation_and_fp32_tracking():
    # full benchmark size (N=4, 64^3 x 6 = 1,572,864 tets, 16 slabs): the conservative strong form conserves the
    # integral of u exactly on the periodic mesh; the FP32 run tracks the FP64 run
    el = d.Element(4)
    w = el.MassMatrix.sum(axis=0)  # integral weights of the reference element (J is constant per tet)
    P = BurgersProblem(4, 64, 16, np.float64, "modes", conservative=1)
    m0 = float(np.sum(P.u0.reshape(P.K, -1) @ w))
    P.run_stages(5)
    u = P.get("u")
    m1 = float(np.sum(u.reshape(P.K, -1) @ w))
    assert abs(m1 - m0) / abs(m0) < 1e-12
    assert np.all(np.isfinite(u))
    P.free()
    A = BurgersProblem(4, 64, 16, np.float64, "modes")
    A.run_stages(10)
    ua = A.get("u")
    A.free()
    B = BurgersProblem(4, 64, 16, np.float32, "modes")
    B.run_stages(10)
    ub = B.get("u")
    B.free()
    assert rel_l2(ub, ua) < 1e-6
