"""Gambit neutral mesh reader (dgk_read_gambit) and the FaceConnector on the reference's partitioned cube, on the
host (no GPU).

The fixture tests/golden/cube_partitioned.json holds the DGKernel mesh mesh/cube-partitioned.neu (565 tets,
element groups p1..p4 and one material group, one boundary set) as lists; the tests write it back as a Gambit
file and read it with the library and with the oracle's restatement of ReadGambitNeutral
(mesh/readers/gambit_reader.go:13-338).  Partition ids are taken from the group names as the reference does
(1..4, partition 0 empty: utils/face_connector.go:58-64 sizes the partition set by the largest id).  Integer
results are compared exactly.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from dgkernel_b200 import _lib
from dgkernel_b200 import mesh as M
from oracle import gambit_ref as G
from oracle import gonudg_ref as g

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cube_partitioned.json")


@pytest.fixture(scope="module")
def cube_file(tmp_path_factory):
    with open(FIX) as f:
        fx = json.load(f)
    path = str(tmp_path_factory.mktemp("neu") / "cube-partitioned.neu")
    G.write(path, fx["nodes"], fx["elements"], fx["groups"], fx["bcs"], "partitioned cube")
    return path


def _same(a, b):
    for k in ("VX", "VY", "VZ", "EToV", "bfaces"):
        assert np.array_equal(a[k], b[k]), k
    assert (a["EToP"] is None) == (b["EToP"] is None)
    if a["EToP"] is not None:
        assert np.array_equal(a["EToP"], b["EToP"])


def test_reader_matches_oracle_on_partitioned_cube(cube_file):
    got = M.read_gambit(cube_file)
    _same(got, G.read(cube_file))
    assert got["EToV"].shape == (565, 4) and len(got["VX"]) == 175
    ids, counts = np.unique(got["EToP"], return_counts=True)
    # gambit_reader_file_test.go: four partitions p1..p4 of 142, 141, 141, 141 elements, largest id 4
    assert ids.tolist() == [1, 2, 3, 4] and counts.tolist() == [142, 141, 141, 141]
    assert got["bfaces"].shape == (42, 3) and set(got["bfaces"][:, 1]) <= {0, 1, 2, 3}


def _kuhn_file(path, groups, shuffle_seed=5):
    """A 2^3 x 6 Kuhn cube written as a Gambit file with shuffled 1-based node and element ids."""
    VX, VY, VZ, EToV, _, _ = M.kuhn_mesh(2, 1, 0.0, 1.0)
    rng = np.random.default_rng(shuffle_seed)
    nid = rng.permutation(len(VX)) + 10
    eid = rng.permutation(EToV.shape[0]) + 3
    nodes = [(int(nid[i]), VX[i], VY[i], VZ[i]) for i in range(len(VX))]
    elements = [(int(eid[k]), *[int(nid[v]) for v in EToV[k]]) for k in range(EToV.shape[0])]
    grp = [(t, name, [int(eid[k]) for k in sel]) for t, name, sel in groups(EToV.shape[0])]
    G.write(path, nodes, elements, grp, [("wall", [(int(eid[0]), 2), (int(eid[5]), 4)])])
    return EToV


def test_reader_two_partition_groups(tmp_path):
    p = str(tmp_path / "two.neu")
    EToV = _kuhn_file(p, lambda K: [(1, "p1", range(0, K, 2)), (2, "p2", range(1, K, 2))])
    got = M.read_gambit(p)
    _same(got, G.read(p))
    assert np.array_equal(got["EToV"], EToV)
    assert got["EToP"].tolist() == [1 + (k % 2) for k in range(EToV.shape[0])]
    assert got["bfaces"].tolist() == [[0, 1, 0], [5, 3, 0]]


def test_reader_single_group_has_no_partitions(tmp_path):
    p = str(tmp_path / "one.neu")
    _kuhn_file(p, lambda K: [(1, "Material group 1", range(K))])
    got = M.read_gambit(p)
    assert got["EToP"] is None
    _same(got, G.read(p))


def test_reader_errors(tmp_path):
    L = _lib.lib()
    counts = np.zeros(4, dtype=np.int64)
    cp = counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    assert L.dgk_read_gambit(str(tmp_path / "missing.neu").encode(), cp, None, None, None, None, None, None) != 0
    p = tmp_path / "hex.neu"
    G.write(str(p), [(1, 0, 0, 0), (2, 1, 0, 0), (3, 0, 1, 0), (4, 0, 0, 1)], [(1, 1, 2, 3, 4)],
            [(1, "g", [1])], [])
    p.write_text(p.read_text().replace("       1  6  4 ", "       1  4  8 "))
    assert L.dgk_read_gambit(str(p).encode(), cp, None, None, None, None, None, None) == _lib.ERR_INVALID
    assert b"tetrahedra" in L.dgk_global_error()


@pytest.mark.parametrize("N", [1, 2, 4])
def test_face_connector_bit_exact_on_partitioned_cube(cube_file, N):
    """tiConnect3D, BuildMaps3D (not periodic) and the FaceConnector pick/place lists of the cube with the
    reference's raw partition ids (partition 0 empty): library against oracle, every (src, dst) pair."""
    m = G.read(cube_file)
    el = g.ref_element(N)
    EToE, EToF = M.ti_connect3d(m["EToV"])
    oE, oF = g.ti_connect3d(m["EToV"])
    assert np.array_equal(EToE, oE) and np.array_equal(EToF, oF)
    X, Y, Z = g.node_coords(el, m["VX"], m["VY"], m["VZ"], m["EToV"])
    _, vmapP, _, mapB = g.build_maps3d(el, X, Y, Z, oE, oF)
    assert len(mapB) > 0
    K = m["EToV"].shape[0]
    fc = M.FaceConnector(K, 4, el.Nfp, el.Np, vmapP, m["EToP"])
    ofc = g.face_connector(K, 4, el.Nfp, el.Np, vmapP, m["EToP"])
    assert fc.NumPartitions == ofc.nparts == 5 and fc.ElemsPerPartition == [0, 142, 141, 141, 141]
    for a in range(5):
        for b in range(5):
            assert np.array_equal(fc.GetPickIndices(a, b), ofc.pick[a][b])
            assert np.array_equal(fc.GetPlaceIndices(b, a), ofc.place[b][a])
    g.face_connector_verify(ofc, el.Np, 4, el.Nfp)


@pytest.mark.parametrize("N", [1, 2, 3])
def test_oracle_physical_derivative_on_partitioned_cube(cube_file, N):
    """The reference's TestTetNudgPhysicalDerivative (tetnudg/tet_nudg_mesh_physical_derivative_test.go:747-919)
    on the oracle: u = x^N + y^N + z^N on the 565-tet partitioned cube, elements stored partition by partition,
    the volume derivative (Dr, Ds, Dt, then the geometric factors) per partition against the analytic
    N x^(N-1), N y^(N-1), N z^(N-1) at the reference's 1e-8 (:911-918).  The nodal derivative is exact for degree
    N on straight-sided tetrahedra, so what is left is rounding."""
    from oracle import burgers_ref as b
    from oracle import oracle as O

    m = G.read(cube_file)
    ref = b.MeshProblem(N, m["VX"], m["VY"], m["VZ"], m["EToV"], m["EToP"], "sine")
    assert ref.Kpart == [142, 141, 141, 141]
    X, Y, Z = ref.X, ref.Y, ref.Z
    U = X ** N + Y ** N + Z ** N
    geo = [getattr(ref.geo, n) for n in ("rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz")]
    dx, dy, dz = O.differentiate(ref.el, ref.Kpart, U, geo, threads=2)
    for got, c in ((dx, X), (dy, Y), (dz, Z)):
        want = (N * c ** (N - 1)).reshape(-1)
        err = np.max(np.abs(got - want))
        assert err < 1e-8, (N, err)
