"""Parity of the mixed-precision stage (rhsStageMixed) with the FP64 oracle, through the runner / C ABI.

The mixed stage keeps the state as a compensated FP32 pair and evaluates the element-local products in FP32
after subtracting each element's linear interpolant, so it does not reproduce FP64 bit for bit.  Stated
bounds, relative L2 against the oracle's FP64 state after the given number of LSERK4 stages:
  * MIXED_TOL = 1e-7 for smooth random-mode fields over 10 stages (measured about 1e-8 .. 3e-8);
  * the same bound for the conservative form and for partitions of ragged size (K per partition not a
    multiple of the 32-element slot, so the last slot's copies end mid-way through a 16-byte word);
  * ORDER5_TOL = 3e-7 at order 5, whose derivative and LIFT entries are 3-4x larger than order 4's
    (measured about 1.1e-7).
The compact geometry and connectivity are checked exactly on the host (test_mixed_host.py) and, here, by
a mixed stage that matches the oracle on a mesh with several partitions.
"""
import numpy as np
import pytest

from dgkernel_b200.burgers import BurgersProblem, MIXED
from oracle import burgers_ref as b
from oracle import oracle as O

from conftest import rel_l2

pytestmark = pytest.mark.gpu
MIXED_TOL = 1e-7
ORDER5_TOL = 3e-7


def _oracle_run(N, n, nslab, u0, dt, nstages, conservative=0):
    ref = b.Problem(N, n, nslab, "sine")
    rs = O.RunState(ref)
    u = np.ascontiguousarray(u0, dtype=np.float64).copy()
    resu = np.zeros_like(u)
    rs.run(u, resu, dt, nstages, conservative=conservative, threads=4)
    return u


@pytest.mark.parametrize("N,n,nslab", [(2, 4, 2), (3, 4, 4), (4, 4, 2), (4, 5, 5), (1, 6, 3)])
def test_mixed_stage_matches_fp64_oracle(N, n, nslab):
    P = BurgersProblem(N, n, nslab, MIXED, "modes")
    u0 = P.u0.copy()
    P.run_stages(10)
    got = P.get("u")
    want = _oracle_run(N, n, nslab, u0, P.dt, 10)
    err = rel_l2(got, want)
    assert err < MIXED_TOL, err
    assert np.max(np.abs(got - want)) < 20 * MIXED_TOL
    P.free()


def test_mixed_stage_conservative_form():
    P = BurgersProblem(4, 4, 2, MIXED, "modes", conservative=1)
    u0 = P.u0.copy()
    P.run_stages(10)
    got = P.get("u")
    want = _oracle_run(4, 4, 2, u0, P.dt, 10, conservative=1)
    assert rel_l2(got, want) < MIXED_TOL
    P.free()


def test_mixed_stage_tracks_fp64_gpu_path():
    """Same u0 through the plain FP64 kernel and the mixed kernel: agreement within the mixed bound."""
    A = BurgersProblem(4, 8, 4, np.float64, "modes")
    B = BurgersProblem(4, 8, 4, MIXED, "modes")
    assert rel_l2(B.u0, A.u0) < 1e-15
    A.run_stages(25)
    B.run_stages(25)
    assert rel_l2(B.get("u"), A.get("u")) < MIXED_TOL
    A.free()
    B.free()


@pytest.mark.parametrize("warps,ring", [(11, 2), (11, 6), (8, 3), (4, 2)])
def test_mixed_launch_shapes_agree_bitwise(warps, ring):
    """Ring depths below the consumer-warp count make warps reuse ring slots out of step with each other; every
    launch shape must give the same bits as the default one (the per-element arithmetic is the same)."""
    A = BurgersProblem(3, 16, 4, MIXED, "modes")
    B = BurgersProblem(3, 16, 4, MIXED, "modes", warps=warps, ring=ring)
    A.run_stages(10)
    B.run_stages(10)
    assert np.array_equal(A.get("u"), B.get("u"))
    A.free()
    B.free()


@pytest.mark.parametrize("conservative", [0, 1])
def test_mixed_stage_order5_matches_fp64_oracle(conservative):
    P = BurgersProblem(5, 4, 2, MIXED, "modes", conservative=conservative)
    u0 = P.u0.copy()
    P.run_stages(10)
    want = _oracle_run(5, 4, 2, u0, P.dt, 10, conservative=conservative)
    assert rel_l2(P.get("u"), want) < ORDER5_TOL
    P.free()
