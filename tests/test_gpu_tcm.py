"""Parity of the tensor-core mixed stage (rhsStageMixed with mma=1: the element-local products as GEMMs on
tcgen05 with three-part BF16 operands and FP32 accumulation) with the FP64 oracle, through the runner / C ABI.

Bounds, relative L2 against the oracle's FP64 state after 10 LSERK4 stages of smooth random-mode fields:
MMA_TOL = 1e-7, the bound of the FP32-product mixed stage (the three-part split keeps about 24 significant
bits of every operand; measured 3.5e-8 .. 6.7e-8); the same for the conservative form, for both launch shapes
(2 and 4 threads per element) and for partitions whose element counts are not multiples of the 128-element
tile (partial tiles, and slot copies that end inside a 16-byte word).
"""
import numpy as np
import pytest

from dgkernel_b200.burgers import BurgersProblem, MIXED
from oracle import burgers_ref as b
from oracle import oracle as O

from conftest import rel_l2

pytestmark = pytest.mark.gpu
MMA_TOL = 1e-7


def _oracle_run(N, n, nslab, u0, dt, nstages, conservative=0):
    ref = b.Problem(N, n, nslab, "sine")
    rs = O.RunState(ref)
    u = np.ascontiguousarray(u0, dtype=np.float64).copy()
    resu = np.zeros_like(u)
    rs.run(u, resu, dt, nstages, conservative=conservative, threads=4)
    return u


@pytest.mark.parametrize("N,n,nslab,warps", [(4, 4, 2, 16), (4, 4, 2, 8), (3, 5, 5, 16), (2, 6, 3, 16),
                                             (1, 6, 2, 8), (4, 7, 7, 16)])
def test_tcm_stage_matches_fp64_oracle(N, n, nslab, warps):
    P = BurgersProblem(N, n, nslab, MIXED, "modes", mma=True, warps=warps)
    u0 = P.u0.copy()
    P.run_stages(10)
    got = P.get("u")
    want = _oracle_run(N, n, nslab, u0, P.dt, 10)
    err = rel_l2(got, want)
    print(f"order {N} n {n} warps {warps}: relative L2 {err:.3e}")
    assert err < MMA_TOL, err
    P.free()


def test_tcm_stage_conservative_form():
    P = BurgersProblem(4, 5, 5, MIXED, "modes", conservative=1, mma=True)
    u0 = P.u0.copy()
    P.run_stages(10)
    want = _oracle_run(4, 5, 5, u0, P.dt, 10, conservative=1)
    assert rel_l2(P.get("u"), want) < MMA_TOL
    P.free()


def test_tcm_stage_tracks_simt_mixed_stage():
    """Many tiles per CTA (16^3 x 6 = 24,576 elements, 192 tiles): the tensor-core and FP32-FMA forms of the
    same stage stay within the mixed bound of each other over 25 stages."""
    A = BurgersProblem(4, 16, 4, MIXED, "modes")
    B = BurgersProblem(4, 16, 4, MIXED, "modes", mma=True)
    A.run_stages(25)
    B.run_stages(25)
    assert np.isfinite(B.get("u")).all()
    assert rel_l2(B.get("u"), A.get("u")) < MMA_TOL
    A.free()
    B.free()


def test_tcm_stage_matches_three_part_restatement():
    """One stage from resu = 0: the GPU residual dt*rhs against the numpy restatement of the same three-part
    split algorithm (oracle/precision_ref.py, exact products and FP64 sums): they differ only by the tensor
    cores' FP32 accumulation over rows whose terms cancel, and FP32 rounding order (bound 3e-6 relative L2;
    measured 1.4e-6; the restatement itself is 1.6e-7 from the FP64 right-hand side, test_split_host.py)."""
    from oracle import precision_ref as PR
    P = BurgersProblem(4, 4, 1, MIXED, "modes", mma=True)
    hi0, lo0 = P.get("uhi").copy(), P.get("ulo").copy()
    P.run_stages(1)
    resu = P.get("resu").astype(np.float64)
    ref = b.Problem(4, 4, 1, "modes")
    want = P.dt * PR.rhs(ref, hi0, lo0, parts=3).astype(np.float64).reshape(-1)
    err = rel_l2(resu, want)
    print(f"tensor-core mixed stage vs three-part restatement: {err:.3e}")
    assert err < 3e-6, err
    P.free()


@pytest.mark.parametrize("form", ["fp64", "mixed_tc"])
def test_benchmark_shaped_mesh_pinned_to_oracle(form):
    """The benchmark's shape at a size the oracle runs in seconds: order 4, 16 x-slab partitions of a 16^3 x 6
    mesh (24,576 tets, 192 tensor-core tiles), the random-mode u0 of the benchmark, 10 LSERK4 stages through
    the runner, against the oracle's own setup and run: plain FP64 stage <= 1e-12, tensor-core mixed stage
    <= MMA_TOL."""
    kw = {"mma": True} if form == "mixed_tc" else {}
    P = BurgersProblem(4, 16, 16, MIXED if form == "mixed_tc" else np.float64, "modes", **kw)
    ref = b.Problem(4, 16, 16, "modes")
    assert rel_l2(P.u0, ref.u0) < 1e-15
    rs = O.RunState(ref)
    u = np.ascontiguousarray(ref.u0, dtype=np.float64).copy()
    resu = np.zeros_like(u)
    rs.run(u, resu, P.dt, 10, threads=8)
    P.run_stages(10)
    err = rel_l2(P.get("u"), u)
    print(f"{form}: relative L2 vs oracle after 10 stages at 16^3 x 6, 16 slabs: {err:.3e}")
    assert err < (1e-12 if form == "fp64" else MMA_TOL), err
    P.free()
