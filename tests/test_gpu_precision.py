"""Precision form on the tensor cores (rhsStageMixed with tensor=1, orders 4..7): both element-local products
as exact integer-digit GEMMs (tcgen05 kind::i8, six digits per operand, levels joined in FP64), compensated
FP32 state, through the runner / C ABI.

Bounds:
  * against the numpy restatement of the same algorithm (oracle/precision_ref.py stage_exact with the library's
    own reference matrices: the same digits, exact int64 digit products, the same FP64 roundings, the kernel's
    element arithmetic being contraction-free) after two stages: the FP32 residual within RESU_TOL = 1e-8
    relative L2 and the FP64 state u = hi + lo within STATE_TOL = 1e-12, both with the library's own metric and
    face arrays (whose FP32-rounded sums the stage uses);
  * against the FP64 oracle after 10 LSERK4 stages: ORACLE_TOL[N], twice the measured error on a B200 (4.4e-10,
    2.2e-10, 6.0e-10, 8.7e-10 at orders 4..7: the ~47-bit products on the reference's ill-conditioned node set,
    plus the FP32 residual).
"""
from types import SimpleNamespace

import numpy as np
import pytest

from dgkernel_b200.burgers import BurgersProblem, MIXED, RK4A, RK4B
from oracle import burgers_ref as b
from oracle import oracle as O
from oracle import precision_ref as PR

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def library_geometry(P):
    """The problem's own FP64 metric and face arrays, shaped as the oracle's Geometry fields."""
    K, Np, NF = P.K, P.el.Np, 4 * P.el.Nfp
    names = {"rx": "Rx", "ry": "Ry", "rz": "Rz", "sx": "Sx", "sy": "Sy", "sz": "Sz", "tx": "Tx", "ty": "Ty",
             "tz": "Tz"}
    d = {k: P.get(v).reshape(K, Np) for k, v in names.items()}
    d.update({k: P.get(k).reshape(K, NF) for k in ("nx", "ny", "nz", "Fscale")})
    return SimpleNamespace(**d)
RESU_TOL = 1e-8
STATE_TOL = 1e-12
ORACLE_TOL = {4: 9e-10, 5: 4.5e-10, 6: 1.2e-9, 7: 1.8e-9}


@pytest.mark.parametrize("N,n,nslab,u0,cons", [(4, 4, 2, "modes", 0), (5, 3, 3, "smooth", 0), (6, 3, 1, "smooth", 0),
                                                (7, 3, 3, "smooth", 0), (7, 4, 1, "smooth", 1), (5, 5, 5, "modes", 1)])
def test_precision_stage_matches_exact_restatement(N, n, nslab, u0, cons):
    P = BurgersProblem(N, n, nslab, MIXED, u0, tensor=True, conservative=cons)
    ref = b.Problem(N, n, nslab, u0)
    hi, lo = P.get("uhi").copy(), P.get("ulo").copy()
    resu = np.zeros_like(hi)
    geo = library_geometry(P)
    for s in range(2):
        hi, lo, resu = PR.stage_exact(ref, hi, lo, resu, RK4A[s], RK4B[s], P.dt, 6, cons, el=P.el, geo=geo)
    P.run_stages(2)
    e_u = rel_l2(P.get("uhi").astype(np.float64) + P.get("ulo"), hi.astype(np.float64) + lo)
    e_r = rel_l2(P.get("resu"), resu)
    print(f"order {N} n {n} cons {cons}: state {e_u:.3e}, residual {e_r:.3e} vs restatement")
    assert e_u < STATE_TOL and e_r < RESU_TOL, (e_u, e_r)
    P.free()


@pytest.mark.parametrize("N,n,nslab,u0", [(4, 4, 2, "modes"), (5, 4, 2, "smooth"), (6, 3, 3, "smooth"),
                                          (7, 3, 1, "smooth")])
def test_precision_stage_matches_fp64_oracle(N, n, nslab, u0):
    P = BurgersProblem(N, n, nslab, MIXED, u0, tensor=True)
    u0v = P.u0.copy()
    P.run_stages(10)
    got = P.get("u")
    ref = b.Problem(N, n, nslab, u0)
    u = np.ascontiguousarray(u0v, dtype=np.float64).copy()
    resu = np.zeros_like(u)
    O.RunState(ref).run(u, resu, P.dt, 10, threads=4)
    err = rel_l2(got, u)
    print(f"order {N} n {n}: relative L2 vs FP64 oracle after 10 stages {err:.3e}")
    assert np.all(np.isfinite(got)) and err < ORACLE_TOL[N], err
    P.free()


def test_precision_stage_agrees_with_tensor_core_mixed_stage():
    """Order 4, many tiles (16^3 x 6 = 24,576 elements, 768 tiles of 32): the exact-digit form and the
    three-part BF16 form of the mixed stage stay within the mixed bound of each other over 25 stages."""
    A = BurgersProblem(4, 16, 4, MIXED, "modes", tensor=True)
    B = BurgersProblem(4, 16, 4, MIXED, "modes", mma=True)
    A.run_stages(25)
    B.run_stages(25)
    assert rel_l2(A.get("u"), B.get("u")) < 1e-7
    A.free()
    B.free()
