"""The oracle against the reference's own golden vectors and property tests (CPU).

Pins: JacobiGL nodes (element/library/gonudg/jacobi_quadrature_test.go:9-136), JacobiP values
(jacobip_test.go:8-92), V*Vinv = I (startup3d_test.go:11-108), metric identities (normals3d_test.go:106-198),
LIFT properties (lift3d_test.go:215-300), tiConnect3D on the 6-tet cube (ticonnect3d_test.go:110-156), and the
FaceConnector element-ID exchange (utils/face_connector_test.go:178-466).
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import gonudg_ref as g

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.json")))


@pytest.mark.parametrize("case", GOLD["jacobi_gl"], ids=lambda c: c["name"])
def test_jacobi_gl_golden(case):
    x = g.jacobi_gl(case["alpha"], case["beta"], case["N"])
    assert len(x) == len(case["expected"])
    assert np.max(np.abs(x - np.array(case["expected"]))) <= case["tol"]


@pytest.mark.parametrize("case", GOLD["jacobi_p"], ids=lambda c: f"a{c['alpha']}b{c['beta']}n{c['N']}")
def test_jacobi_p_golden(case):
    p = g.jacobi_p(np.array(case["x"]), case["alpha"], case["beta"], case["N"])
    assert np.max(np.abs(p - case["value"])) <= case["tol"]


def test_simplex3dp_constant_mode():
    v = g.simplex3dp(np.array([-1.0]), np.array([-1.0]), np.array([-1.0]), 0, 0, 0)
    assert abs(v[0] - GOLD["simplex3dp_000"]) < 1e-10


def test_jacobi_gq_weights_sum_and_symmetry():
    for n in range(0, 6):
        x, w = g.jacobi_gq(0.0, 0.0, n)
        assert abs(w.sum() - 2.0) < 1e-13
        assert np.max(np.abs(x + x[::-1])) < 1e-13


@pytest.mark.parametrize("N", [1, 2, 3, 4])
def test_vandermonde_inverse_and_dims(N):
    el = g.ref_element(N)
    assert el.Np == (N + 1) * (N + 2) * (N + 3) // 6 and el.Nfp == (N + 1) * (N + 2) // 2
    assert el.V.shape == (el.Np, el.Np) and el.LIFT.shape == (el.Np, 4 * el.Nfp)
    assert np.max(np.abs(el.V @ el.Vinv - np.eye(el.Np))) < 1e-10
    assert el.Fmask.shape == (4, el.Nfp)


def _single_tet(N, verts):
    el = g.ref_element(N)
    VX, VY, VZ = (np.array([v[i] for v in verts], float) for i in range(3))
    X, Y, Z = g.node_coords(el, VX, VY, VZ, [[0, 1, 2, 3]])
    return el, X, Y, Z


@pytest.mark.parametrize("N", [1, 2, 3, 4])
def test_polynomial_derivative_exact(N):
    # tetnudg/tet_nudg_mesh_physical_derivative_test.go:747-919: d/dx (x^N + y^N + z^N) exact to 1e-8
    el, X, Y, Z = _single_tet(N, [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    geo = g.geometric_factors(el, X, Y, Z)
    U = X ** N + Y ** N + Z ** N
    Ur, Us, Ut = U @ el.Dr.T, U @ el.Ds.T, U @ el.Dt.T
    dudx = geo.rx * Ur + geo.sx * Us + geo.tx * Ut
    assert np.max(np.abs(dudx - N * X ** (N - 1))) < 1e-8


def test_metric_identities_rotated_scaled():
    a, s = math.pi / 6, 2.0
    base = [[-1, -1, -1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]]
    verts = [[s * (math.cos(a) * v[0] - math.sin(a) * v[1]), s * (math.sin(a) * v[0] + math.cos(a) * v[1]), s * v[2]]
             for v in base]
    el, X, Y, Z = _single_tet(3, verts)
    geo = g.geometric_factors(el, X, Y, Z)
    xr, xs, xt = X @ el.Dr.T, X @ el.Ds.T, X @ el.Dt.T
    yr, ys, yt = Y @ el.Dr.T, Y @ el.Ds.T, Y @ el.Dt.T
    zr, zs, zt = Z @ el.Dr.T, Z @ el.Ds.T, Z @ el.Dt.T
    assert np.max(np.abs(geo.rx * xr + geo.ry * yr + geo.rz * zr - 1)) < 1e-10
    assert np.max(np.abs(geo.rx * xs + geo.ry * ys + geo.rz * zs)) < 1e-10
    assert np.max(np.abs(geo.sx * xs + geo.sy * ys + geo.sz * zs - 1)) < 1e-10
    assert np.max(np.abs(geo.tx * xt + geo.ty * yt + geo.tz * zt - 1)) < 1e-10


def test_normals_unit_and_outward():
    el, X, Y, Z = _single_tet(2, [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    geo = g.geometric_factors(el, X, Y, Z)
    mag = np.sqrt(geo.nx ** 2 + geo.ny ** 2 + geo.nz ** 2)
    assert np.max(np.abs(mag - 1)) < 1e-12
    cx, cy, cz = X.mean(), Y.mean(), Z.mean()
    fm = el.Fmask.reshape(-1)
    dot = (X[0, fm] - cx) * geo.nx[0] + (Y[0, fm] - cy) * geo.ny[0] + (Z[0, fm] - cz) * geo.nz[0]
    assert np.all(dot > 0)


def test_lift_constant_and_face_consistency():
    el = g.ref_element(3)
    lifted = el.LIFT @ np.ones(4 * el.Nfp)
    assert np.max(np.abs(lifted)) > 1e-10
    for f in range(4):
        assert np.all(np.abs(lifted[el.Fmask[f]]) > 1e-10)


def _cube():
    m = GOLD["meshes"]
    nodes = np.array(m["cube_nodes"], float)
    return nodes, np.array(m["cube_tets"], dtype=np.int64)


def test_ticonnect_cube_boundary_and_reciprocity():
    _, tets = _cube()
    E, F = g.ti_connect3d(tets)
    assert int(np.sum(E == np.arange(len(tets))[:, None])) == 12
    for e in range(len(tets)):
        for f in range(4):
            assert E[E[e, f], F[e, f]] == e and F[E[e, f], F[e, f]] == f


def _fake_vmapP(K, Nfp, Np, E, F):
    # the deliberately simple face map of utils/face_connector_test.go:87-110
    v = np.zeros(K * 4 * Nfp, dtype=np.int64)
    for e in range(K):
        for f in range(4):
            for fp in range(Nfp):
                v[e * 4 * Nfp + f * Nfp + fp] = E[e, f] * Np + (F[e, f] * Nfp + fp) % Np
    return v


@pytest.mark.parametrize("EToP", [[0] * 6, [0, 0, 0, 1, 1, 1]])
def test_face_connector_element_id_exchange(EToP):
    _, tets = _cube()
    K, Nfp, Np = len(tets), 3, 4
    E, F = g.ti_connect3d(tets)
    fc = g.face_connector(K, 4, Nfp, Np, _fake_vmapP(K, Nfp, Np, E, F), EToP)
    g.face_connector_verify(fc, Np, 4, Nfp)
    sols = [np.repeat(fc.local_to_global[p].astype(float), Np) for p in range(fc.nparts)]
    pb = g.simulate_face_exchange(fc, sols, 4, Nfp)
    for p in range(fc.nparts):
        for le, ge in enumerate(fc.local_to_global[p]):
            for f in range(4):
                assert np.all(pb[p][le * 4 * Nfp + f * Nfp:(le * 4 + f + 1) * Nfp] == E[ge, f])
    if fc.nparts == 2:
        assert len(fc.pick[0][1]) and len(fc.pick[1][0])


def test_periodic_maps_have_no_boundary():
    from oracle import burgers_ref as b
    p = b.Problem(1, 3, 1)
    assert len(p.mapB) == 0
    g.face_connector_verify(p.fc, p.el.Np, 4, p.el.Nfp)
