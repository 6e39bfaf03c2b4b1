"""The reference's partitioned cube (mesh/cube-partitioned.neu: 565 tets in element groups p1..p4, faces on the
cube's boundary without a neighbour) through the library's Gambit reader and the stage kernels, against the
oracle.  Elements are stored partition by partition; boundary faces keep VmapP = VmapM
(element/library/gonudg/buildmaps3d.go:34).  Bounds: VmapP bit-exact; FP64 stage <= 1e-12 relative L2 after 10
LSERK4 stages at orders 1..4; the mixed forms within their stated bounds of the oracle's FP64 run (FP32-FMA
and three-part BF16 tensor-core products 1e-7, exact-digit precision form 8e-10 at order 4, twice its measured
3.9e-10)."""
import json
import os

import numpy as np
import pytest

from dgkernel_b200 import mesh as M
from dgkernel_b200.burgers import BurgersMesh, MIXED
from oracle import burgers_ref as b
from oracle import gambit_ref as G
from oracle import oracle as O

from conftest import rel_l2

pytestmark = pytest.mark.gpu
FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cube_partitioned.json")


@pytest.fixture(scope="module")
def cube(tmp_path_factory):
    with open(FIX) as f:
        fx = json.load(f)
    path = str(tmp_path_factory.mktemp("neu") / "cube-partitioned.neu")
    G.write(path, fx["nodes"], fx["elements"], fx["groups"], fx["bcs"], "partitioned cube")
    return M.read_gambit(path)


def _oracle(ref, u0, dt, nst, conservative=0):
    u = np.ascontiguousarray(u0, dtype=np.float64).copy()
    resu = np.zeros_like(u)
    O.RunState(ref).run(u, resu, dt, nst, conservative=conservative, threads=4)
    return u


@pytest.mark.parametrize("N", [1, 2, 3, 4])
def test_partitioned_cube_fp64_stages_match_oracle(cube, N):
    P = BurgersMesh(N, cube["VX"], cube["VY"], cube["VZ"], cube["EToV"], cube["EToP"], np.float64, "sine")
    ref = b.MeshProblem(N, cube["VX"], cube["VY"], cube["VZ"], cube["EToV"], cube["EToP"], "sine")
    assert P.Kpart == ref.Kpart == [142, 141, 141, 141] and P.part_ids.tolist() == [1, 2, 3, 4]
    assert np.array_equal(P.order, ref.order)
    assert np.array_equal(P.vmapP, ref.vmapP)
    assert abs(P.dt - ref.dt) < 1e-14 * ref.dt  # h_min from GPU and numpy node coordinates
    u0 = P.u0.copy()
    assert rel_l2(u0, ref.u0) < 1e-15
    P.run_stages(10)
    err = rel_l2(P.get("u"), _oracle(ref, u0, P.dt, 10))
    print(f"order {N}: relative L2 vs oracle {err:.3e}")
    assert err < 1e-12, err
    P.free()


@pytest.mark.parametrize("form", ["mixed", "mixed_tc", "precision"])
def test_partitioned_cube_mixed_forms(cube, form):
    kw = {"mixed": {}, "mixed_tc": {"mma": True}, "precision": {"tensor": True}}[form]
    P = BurgersMesh(4, cube["VX"], cube["VY"], cube["VZ"], cube["EToV"], cube["EToP"], MIXED, "sine", **kw)
    ref = b.MeshProblem(4, cube["VX"], cube["VY"], cube["VZ"], cube["EToV"], cube["EToP"], "sine")
    u0 = P.u0.copy()
    P.run_stages(10)
    err = rel_l2(P.get("u"), _oracle(ref, u0, P.dt, 10))
    print(f"{form}: relative L2 vs oracle {err:.3e}")
    assert err < (8e-10 if form == "precision" else 1e-7), err
    P.free()
