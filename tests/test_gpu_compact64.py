"""The FP64 stage on the compact layout (rhsStage compact=1), through the runner / C ABI.

Same FP64 tensor-path arithmetic as the plain stage; only the layout differs: per-element geometry (node-0
metrics, per-face normals and Fscale, checked constant over each straight-sided element) and the compact
connectivity (neighbour base and face-order code per face) instead of per-node metrics, per-point face arrays
and the gather map.  Bounds: 10 LSERK4 stages against the FP64 oracle at 1e-12 relative L2 (the plain
stage's bar), and against the plain FP64 stage at 1e-13 (the per-node metrics of a straight-sided element agree
to rounding).
"""
import numpy as np
import pytest

from dgkernel_b200._lib import DGKError
from dgkernel_b200.burgers import BurgersProblem
from oracle import burgers_ref as b
from oracle import oracle as O

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,n,slabs,cons", [(1, 4, 2, 0), (2, 8, 4, 0), (3, 4, 4, 1), (4, 4, 2, 0), (5, 3, 1, 0)])
def test_compact_fp64_stage_matches_oracle_and_plain_stage(N, n, slabs, cons):
    ref = b.Problem(N, n, slabs, "modes")
    P = BurgersProblem(N, n, slabs, np.float64, "modes", compact=True, conservative=cons)
    Q = BurgersProblem(N, n, slabs, np.float64, "modes", conservative=cons)
    assert abs(P.dt - ref.dt) <= 1e-14 * ref.dt
    u = np.ascontiguousarray(ref.u0.reshape(-1)).copy()
    resu = np.zeros_like(u)
    O.RunState(ref).run(u, resu, P.dt, 10, conservative=cons)
    P.run_stages(10)
    Q.run_stages(10)
    assert rel_l2(P.get("u"), u) < 1e-12
    assert rel_l2(P.get("u"), Q.get("u")) < 1e-13
    P.free()
    Q.free()


def test_compact_form_is_fp64_only():
    with pytest.raises(DGKError):
        BurgersProblem(2, 4, 2, np.float32, "modes", compact=True)
