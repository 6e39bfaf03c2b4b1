"""CPU FP64 restatement of the reference's nodal-tetrahedron setup chain (test infrastructure only).

This module is the ORACLE for the setup inputs of the tet-DG right-hand side: it is imported only by
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``, as the checker.  The
product (``dgkernel_b200``) has its own C++/CUDA implementation and never calls into this file.

Every function restates the algorithm of the Go file and line it cites (paths are relative to the
DGKernel project root).  Where the reference calls gonum (v0.16.0) for dense linear algebra
(``mat.Dense.Inverse`` = LAPACK getrf/getri, ``mat.EigenSym`` = LAPACK syev), this restatement calls the
LAPACK-backed numpy equivalents, so results agree with the reference to the last few ulps.

Deliberate restatements of reference quirks (parity is to the reference, not to the textbook):
  * ``evalwarp`` (nodes3d.go:290-324) multiplies the full Lagrange interpolant by (1 - x^2) and pairs the
    descending, negated Gauss-Lobatto nodes with ascending equidistant nodes;
  * ``GetRefMatrices`` (tetnudg/tet_nudg_mesh.go:323-389) names V*V^T "M" and its inverse "Minv".
"""
from __future__ import annotations

import math
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

NFACES = 4
NODETOL = 1e-7  # startup3d.go:80


def np_count(n: int) -> int:
    """Np = (N+1)(N+2)(N+3)/6 (startup3d.go:96)."""
    return (n + 1) * (n + 2) * (n + 3) // 6


def nfp_count(n: int) -> int:
    """Nfp = (N+1)(N+2)/2 (startup3d.go:97)."""
    return (n + 1) * (n + 2) // 2


# --------------------------------------------------------------------------------------------------
# 1-D orthonormal Jacobi polynomials and Gauss quadrature (jacobip.go, jacobi_quadrature.go)
# --------------------------------------------------------------------------------------------------
def jacobi_p(x, alpha: float, beta: float, n: int) -> np.ndarray:
    """Orthonormal Jacobi polynomial P_n^(alpha,beta)(x) by the three-term recurrence (jacobip.go:30-98)."""
    x = np.asarray(x, dtype=np.float64)
    ab = alpha + beta
    ab1 = alpha + beta + 1.0
    a1 = alpha + 1.0
    b1 = beta + 1.0
    gamma0 = math.pow(2.0, ab1) / ab1 * math.gamma(a1) * math.gamma(b1) / math.gamma(ab1)
    p_prev = np.full(x.shape, 1.0 / math.sqrt(gamma0))
    if n == 0:
        return p_prev
    gamma1 = a1 * b1 / (ab + 3.0) * gamma0
    p_cur = ((ab + 2.0) * x / 2.0 + (alpha - beta) / 2.0) * (1.0 / math.sqrt(gamma1))
    if n == 1:
        return p_cur
    aold = 2.0 / (2.0 + ab) * math.sqrt(a1 * b1 / (ab + 3.0))
    for i in range(1, n):
        fi = float(i)
        h1 = 2.0 * fi + ab
        anew = 2.0 / (h1 + 2.0) * math.sqrt((fi + 1.0) * (fi + ab1) * (fi + a1) * (fi + b1) / (h1 + 1.0) / (h1 + 3.0))
        bnew = -(alpha * alpha - beta * beta) / h1 / (h1 + 2.0)
        p_next = 1.0 / anew * (-aold * p_prev + (x - bnew) * p_cur)
        p_prev, p_cur = p_cur, p_next
        aold = anew
    return p_cur


def grad_jacobi_p(x, alpha: float, beta: float, n: int) -> np.ndarray:
    """d/dx P_n = sqrt(n(n+a+b+1)) P_{n-1}^(a+1,b+1) (jacobip.go:107-121)."""
    x = np.asarray(x, dtype=np.float64)
    if n == 0:
        return np.zeros(x.shape)
    return jacobi_p(x, alpha + 1.0, beta + 1.0, n - 1) * math.sqrt(n * (n + alpha + beta + 1.0))


def gamma0(alpha: float, beta: float) -> float:
    """jacobi_quadrature.go:103-108."""
    ab1 = alpha + beta + 1.0
    return math.gamma(alpha + 1.0) * math.gamma(beta + 1.0) * math.pow(2.0, ab1) / ab1 / math.gamma(ab1)


def jacobi_gq(alpha: float, beta: float, n: int):
    """Gauss-Jacobi nodes/weights from the symmetric tridiagonal Jacobi matrix (jacobi_quadrature.go:39-101)."""
    if n == 0:
        return np.array([-(alpha - beta) / (alpha + beta + 2.0)]), np.array([2.0])
    i = np.arange(n + 1, dtype=np.float64)
    h1 = 2.0 * i + alpha + beta
    with np.errstate(divide="ignore", invalid="ignore"):
        d0 = (beta * beta - alpha * alpha) / (h1 * (h1 + 2.0))
    if alpha + beta < 10 * 1e-16:
        d0[0] = 0.0
    ip1 = np.arange(1, n + 1, dtype=np.float64)
    hv = h1[:n]
    d1 = 2.0 / (hv + 2.0) * np.sqrt(ip1 * (ip1 + alpha + beta) * (ip1 + alpha) * (ip1 + beta) / (hv + 1.0) / (hv + 3.0))
    jj = np.diag(d0) + np.diag(d1, 1) + np.diag(d1, -1)
    x, vecs = np.linalg.eigh(jj)
    w = vecs[0, :] * (vecs[0, :] * gamma0(alpha, beta))
    return x, w


def jacobi_gl(alpha: float, beta: float, n: int) -> np.ndarray:
    """Gauss-Lobatto nodes: endpoints plus JacobiGQ(a+1,b+1,N-2) (jacobi_quadrature.go:16-37)."""
    if n == 0:
        return np.array([0.0])
    if n == 1:
        return np.array([-1.0, 1.0])
    xint, _ = jacobi_gq(alpha + 1.0, beta + 1.0, n - 2)
    return np.concatenate(([-1.0], xint, [1.0]))


# --------------------------------------------------------------------------------------------------
# Warp & blend nodes (nodes3d.go) and coordinate maps (xyztorst.go, rsttoabc.go)
# --------------------------------------------------------------------------------------------------
_ALPHASTORE = (0.0000, 0.0000, 0.0000, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577, 1.1603, 1.10153,
               0.6080, 0.4523, 0.8856, 0.8717, 0.9655)  # nodes3d.go:19-23


def equi_nodes3d(p: int):
    """Equidistant nodes, l (r) fastest, n (t) slowest (nodes3d.go:177-205)."""
    if p == 0:
        return np.array([-1.0]), np.array([-1.0]), np.array([-1.0])
    r, s, t = [], [], []
    for n in range(p + 1):
        for m in range(p - n + 1):
            for l in range(p - n - m + 1):
                r.append(-1.0 + 2.0 * l / p)
                s.append(-1.0 + 2.0 * m / p)
                t.append(-1.0 + 2.0 * n / p)
    return np.array(r), np.array(s), np.array(t)


def _evalwarp(p: int, gauss_x: np.ndarray, xnodes: np.ndarray) -> np.ndarray:
    """Lagrange interpolant through (xeq, gaussX - xeq) times (1 - x^2) (nodes3d.go:290-324)."""
    xeq = np.array([-1.0 + 2.0 * i / p for i in range(p + 1)])
    warp = np.zeros_like(xnodes)
    for idx, x in enumerate(xnodes):
        val = 0.0
        for j in range(p + 1):
            lag = 1.0
            for k in range(p + 1):
                if k != j:
                    lag *= (x - xeq[k]) / (xeq[j] - xeq[k])
            val += lag * (gauss_x[j] - xeq[j])
        warp[idx] = val * (1.0 - x * x)
    return warp


def _evalshift(p: int, pval: float, l1, l2, l3):
    """Face warp in the equilateral triangle (nodes3d.go:221-287)."""
    gauss_x = -jacobi_gl(0.0, 0.0, p)
    blend1, blend2, blend3 = l2 * l3, l1 * l3, l1 * l2
    wf1 = _evalwarp(p, gauss_x, l3 - l2) * 4.0
    wf2 = _evalwarp(p, gauss_x, l1 - l3) * 4.0
    wf3 = _evalwarp(p, gauss_x, l2 - l1) * 4.0
    w1 = blend1 * wf1 * (1.0 + pval * pval * l1 * l1)
    w2 = blend2 * wf2 * (1.0 + pval * pval * l2 * l2)
    w3 = blend3 * wf3 * (1.0 + pval * pval * l3 * l3)
    dx = 1.0 * w1 + math.cos(2.0 * math.pi / 3.0) * w2 + math.cos(4.0 * math.pi / 3.0) * w3
    dy = 0.0 * w1 + math.sin(2.0 * math.pi / 3.0) * w2 + math.sin(4.0 * math.pi / 3.0) * w3
    return dx, dy


_SQ3 = math.sqrt(3.0)
_SQ6 = math.sqrt(6.0)
_V1 = np.array([-1.0, -1.0 / _SQ3, -1.0 / _SQ6])
_V2 = np.array([1.0, -1.0 / _SQ3, -1.0 / _SQ6])
_V3 = np.array([0.0, 2.0 / _SQ3, -1.0 / _SQ6])
_V4 = np.array([0.0, 0.0, 3.0 / _SQ6])


def nodes3d(p: int):
    """Warp & blend nodes in the equilateral tetrahedron (nodes3d.go:17-174)."""
    alpha = _ALPHASTORE[p] if 0 <= p < 15 else 1.0
    tol = 1e-10
    r, s, t = equi_nodes3d(p)
    L1 = (1.0 + t) / 2.0
    L2 = (1.0 + s) / 2.0
    L3 = -(1.0 + r + s + t) / 2.0
    L4 = (1.0 + r) / 2.0
    t1 = [_V2 - _V1, _V2 - _V1, _V3 - _V2, _V3 - _V1]
    t2 = [_V3 - 0.5 * (_V1 + _V2), _V4 - 0.5 * (_V1 + _V2), _V4 - 0.5 * (_V2 + _V3), _V4 - 0.5 * (_V1 + _V3)]
    t1 = [v / math.sqrt(float(np.sum(v * v))) for v in t1]
    t2 = [v / math.sqrt(float(np.sum(v * v))) for v in t2]
    X = L3 * _V1[0] + L4 * _V2[0] + L2 * _V3[0] + L1 * _V4[0]
    Y = L3 * _V1[1] + L4 * _V2[1] + L2 * _V3[1] + L1 * _V4[1]
    Z = L3 * _V1[2] + L4 * _V2[2] + L2 * _V3[2] + L1 * _V4[2]
    shift = np.zeros((3, len(r)))
    perms = [(L1, L2, L3, L4), (L2, L1, L3, L4), (L3, L1, L4, L2), (L4, L1, L3, L2)]
    for face, (La, Lb, Lc, Ld) in enumerate(perms):
        w1, w2 = _evalshift(p, alpha, Lb, Lc, Ld)
        blend = Lb * Lc * Ld
        denom = (Lb + 0.5 * La) * (Lc + 0.5 * La) * (Ld + 0.5 * La)
        ok = denom > tol
        blend = np.where(ok, (1.0 + alpha * alpha * La * La) * blend / np.where(ok, denom, 1.0), blend)
        for d in range(3):
            shift[d] += blend * w1 * t1[face][d] + blend * w2 * t2[face][d]
        count = (Lb > tol).astype(int) + (Lc > tol).astype(int) + (Ld > tol).astype(int)
        fix = (La < tol) & (count < 3)
        for d in range(3):
            shift[d] = np.where(fix, w1 * t1[face][d] + w2 * t2[face][d], shift[d])
    return X + shift[0], Y + shift[1], Z + shift[2]


def xyz_to_rst(X, Y, Z):
    """Affine map from the equilateral to the reference tetrahedron (xyztorst.go:8-69)."""
    A = 0.5 * np.column_stack((_V2 - _V1, _V3 - _V1, _V4 - _V1))
    off = 0.5 * (_V2 + _V3 + _V4 - _V1)
    det = (A[0, 0] * (A[1, 1] * A[2, 2] - A[1, 2] * A[2, 1]) - A[0, 1] * (A[1, 0] * A[2, 2] - A[1, 2] * A[2, 0])
           + A[0, 2] * (A[1, 0] * A[2, 1] - A[1, 1] * A[2, 0]))
    inv = np.array([
        [(A[1, 1] * A[2, 2] - A[1, 2] * A[2, 1]) / det, (A[0, 2] * A[2, 1] - A[0, 1] * A[2, 2]) / det,
         (A[0, 1] * A[1, 2] - A[0, 2] * A[1, 1]) / det],
        [(A[1, 2] * A[2, 0] - A[1, 0] * A[2, 2]) / det, (A[0, 0] * A[2, 2] - A[0, 2] * A[2, 0]) / det,
         (A[0, 2] * A[1, 0] - A[0, 0] * A[1, 2]) / det],
        [(A[1, 0] * A[2, 1] - A[1, 1] * A[2, 0]) / det, (A[0, 1] * A[2, 0] - A[0, 0] * A[2, 1]) / det,
         (A[0, 0] * A[1, 1] - A[0, 1] * A[1, 0]) / det]])
    rx, ry, rz = X - off[0], Y - off[1], Z - off[2]
    r = inv[0, 0] * rx + inv[0, 1] * ry + inv[0, 2] * rz
    s = inv[1, 0] * rx + inv[1, 1] * ry + inv[1, 2] * rz
    t = inv[2, 0] * rx + inv[2, 1] * ry + inv[2, 2] * rz
    return r, s, t


def rst_to_abc(r, s, t):
    """Collapsed coordinates with the 1e-12 singular-point guards (rsttoabc.go:7-34)."""
    r, s, t = (np.asarray(v, dtype=np.float64) for v in (r, s, t))
    tol = 1e-12
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(np.abs(s + t) < tol, -1.0, 2.0 * (1.0 + r) / (-s - t) - 1.0)
        b = np.where(np.abs(t - 1.0) < tol, -1.0, 2.0 * (1.0 + s) / (1.0 - t) - 1.0)
    return a, b, t.copy()


# --------------------------------------------------------------------------------------------------
# Orthonormal simplex basis, Vandermonde and differentiation matrices
# --------------------------------------------------------------------------------------------------
def simplex3dp(a, b, c, i: int, j: int, k: int) -> np.ndarray:
    """Orthonormal tet basis function (i,j,k) (simplex3dp.go:15-36)."""
    h1 = jacobi_p(a, 0.0, 0.0, i)
    h2 = jacobi_p(b, float(2 * i + 1), 0.0, j)
    h3 = jacobi_p(c, float(2 * (i + j) + 2), 0.0, k)
    return (2.0 * math.sqrt(2.0) * h1 * h2) * np.power(1.0 - b, float(i)) * (h3 * np.power(1.0 - c, float(i + j)))


def grad_simplex3dp(r, s, t, i: int, j: int, k: int):
    """Gradient of basis function (i,j,k) w.r.t. (r,s,t) (simplex3dp.go:56-118)."""
    a, b, c = rst_to_abc(r, s, t)
    fa, gb, hc = jacobi_p(a, 0, 0, i), jacobi_p(b, 2 * i + 1, 0, j), jacobi_p(c, 2 * (i + j) + 2, 0, k)
    dfa, dgb, dhc = (grad_jacobi_p(a, 0, 0, i), grad_jacobi_p(b, 2 * i + 1, 0, j),
                     grad_jacobi_p(c, 2 * (i + j) + 2, 0, k))
    norm = math.pow(2.0, float(2 * i + j) + 1.5)
    vr = dfa * gb * hc
    if i > 0:
        vr = vr * np.power(0.5 * (1.0 - b), float(i - 1))
    if i + j > 0:
        vr = vr * np.power(0.5 * (1.0 - c), float(i + j - 1))
    vs = 0.5 * (1.0 + a) * vr
    tmp = dgb * np.power(0.5 * (1.0 - b), float(i))
    if i > 0:
        tmp = tmp - (0.5 * i) * gb * np.power(0.5 * (1.0 - b), float(i - 1))
    if i + j > 0:
        tmp = tmp * np.power(0.5 * (1.0 - c), float(i + j - 1))
    tmp = fa * tmp * hc
    vs = vs + tmp
    vt = 0.5 * (1.0 + a) * vr + 0.5 * (1.0 + b) * tmp
    tmp2 = dhc * np.power(0.5 * (1.0 - c), float(i + j))
    if i + j > 0:
        tmp2 = tmp2 - (0.5 * (i + j)) * hc * np.power(0.5 * (1.0 - c), float(i + j - 1))
    tmp2 = fa * gb * tmp2
    tmp2 = tmp2 * np.power(0.5 * (1.0 - b), float(i))
    vt = vt + tmp2
    return vr * norm, vs * norm, vt * norm


def _modes3d(n: int):
    """Mode order i, then j, then k with i+j+k <= N (vandermonde3d.go:24-37)."""
    return [(i, j, k) for i in range(n + 1) for j in range(n - i + 1) for k in range(n - i - j + 1)]


def vandermonde3d(n: int, r, s, t) -> np.ndarray:
    """V[p, m] = phi_m(r_p) (vandermonde3d.go:15-40)."""
    a, b, c = rst_to_abc(r, s, t)
    return np.column_stack([simplex3dp(a, b, c, i, j, k) for (i, j, k) in _modes3d(n)])


def grad_vandermonde3d(n: int, r, s, t):
    """Vr, Vs, Vt (vandermonde3d.go:45-73)."""
    cols = [grad_simplex3dp(r, s, t, i, j, k) for (i, j, k) in _modes3d(n)]
    return (np.column_stack([c[0] for c in cols]), np.column_stack([c[1] for c in cols]),
            np.column_stack([c[2] for c in cols]))


def simplex2dp(R, S, i: int, j: int) -> np.ndarray:
    """Orthonormal triangle basis function (vandermonde2D.go:34-55)."""
    R, S = np.asarray(R, float), np.asarray(S, float)
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(S != 1.0, 2.0 * (1.0 + R) / (1.0 - S) - 1.0, -1.0)
    b = S
    h1 = jacobi_p(a, 0.0, 0.0, i)
    h2 = jacobi_p(b, float(2 * i + 1), 0.0, j)
    tv2 = np.ones_like(b)
    if i > 0:
        tv2 = 1.0 - b
        for _ in range(1, i):
            tv2 = tv2 * (1.0 - b)
    return (1.4142135623730951 * h1 * h2) * tv2


def vandermonde2d(n: int, R, S) -> np.ndarray:
    """vandermonde2D.go:9-31."""
    return np.column_stack([simplex2dp(R, S, i, j) for i in range(n + 1) for j in range(n - i + 1)])


# --------------------------------------------------------------------------------------------------
# Reference element (StartUp3D up to the mesh-independent operators)
# --------------------------------------------------------------------------------------------------
@dataclass
class RefElement:
    N: int
    Np: int
    Nfp: int
    r: np.ndarray
    s: np.ndarray
    t: np.ndarray
    V: np.ndarray
    Vinv: np.ndarray
    MassMatrix: np.ndarray
    Dr: np.ndarray
    Ds: np.ndarray
    Dt: np.ndarray
    LIFT: np.ndarray
    Fmask: np.ndarray  # (4, Nfp) int

    def ref_matrices(self) -> dict:
        """GetRefMatrices naming "<Op>_NudgTet<N>" (tetnudg/tet_nudg_mesh.go:371-389, :234)."""
        sn = f"NudgTet{self.N}"
        M = self.V @ self.V.T  # tet_nudg_mesh.go:323-330 names V*V^T "M"
        return {f"V_{sn}": self.V, f"Vinv_{sn}": self.Vinv, f"M_{sn}": M, f"Minv_{sn}": np.linalg.inv(M),
                f"Dr_{sn}": self.Dr, f"Ds_{sn}": self.Ds, f"Dt_{sn}": self.Dt, f"LIFT_{sn}": self.LIFT}


def build_fmask(r, s, t, tol: float = NODETOL) -> np.ndarray:
    """Face node lists: t=-1, s=-1, r+s+t=-1, r=-1 (startup3d.go:179-209)."""
    masks = [np.nonzero(np.abs(1.0 + t) < tol)[0], np.nonzero(np.abs(1.0 + s) < tol)[0],
             np.nonzero(np.abs(1.0 + r + s + t) < tol)[0], np.nonzero(np.abs(1.0 + r) < tol)[0]]
    return np.array(masks, dtype=np.int64)


def lift3d(n: int, r, s, t, V, fmask) -> np.ndarray:
    """LIFT = V (V^T Emat) with per-face inv(VFace VFace^T) blocks (lift3d.go:9-90)."""
    Np, Nfp = len(r), fmask.shape[1]
    emat = np.zeros((Np, NFACES * Nfp))
    coords = [(r, s), (r, t), (s, t), (s, t)]
    for f in range(NFACES):
        fr, fs = coords[f][0][fmask[f]], coords[f][1][fmask[f]]
        vf = vandermonde2d(n, fr, fs)
        mass_face = np.linalg.inv(vf @ vf.T)
        emat[fmask[f], f * Nfp:(f + 1) * Nfp] = mass_face
    return V @ (V.T @ emat)


def ref_element(n: int) -> RefElement:
    """Mesh-independent part of StartUp3D (startup3d.go:94-118, 158-162)."""
    x1, y1, z1 = nodes3d(n)
    r, s, t = xyz_to_rst(x1, y1, z1)
    V = vandermonde3d(n, r, s, t)
    Vinv = np.linalg.inv(V)
    mass = Vinv.T @ Vinv
    Vr, Vs, Vt = grad_vandermonde3d(n, r, s, t)
    Dr, Ds, Dt = Vr @ Vinv, Vs @ Vinv, Vt @ Vinv
    fmask = build_fmask(r, s, t)
    lift = lift3d(n, r, s, t, V, fmask)
    return RefElement(n, np_count(n), nfp_count(n), r, s, t, V, Vinv, mass, Dr, Ds, Dt, lift, fmask)


# --------------------------------------------------------------------------------------------------
# Physical mesh: node coordinates, geometric factors, normals, Fscale (startup3d.go, normals3d.go)
# --------------------------------------------------------------------------------------------------
def node_coords(el: RefElement, VX, VY, VZ, EToV):
    """Physical node coordinates, element-contiguous (K, Np) (startup3d.go:126-148)."""
    EToV = np.asarray(EToV)
    va, vb, vc, vd = EToV[:, 0], EToV[:, 1], EToV[:, 2], EToV[:, 3]
    r, s, t = el.r[None, :], el.s[None, :], el.t[None, :]

    def m(v):
        v = np.asarray(v, float)
        return 0.5 * (-(1.0 + r + s + t) * v[va][:, None] + (1.0 + r) * v[vb][:, None]
                      + (1.0 + s) * v[vc][:, None] + (1.0 + t) * v[vd][:, None])
    return m(VX), m(VY), m(VZ)


@dataclass
class Geometry:
    J: np.ndarray
    rx: np.ndarray
    ry: np.ndarray
    rz: np.ndarray
    sx: np.ndarray
    sy: np.ndarray
    sz: np.ndarray
    tx: np.ndarray
    ty: np.ndarray
    tz: np.ndarray
    nx: np.ndarray
    ny: np.ndarray
    nz: np.ndarray
    sJ: np.ndarray
    Fscale: np.ndarray


def geometric_factors(el: RefElement, X, Y, Z) -> Geometry:
    """Metric terms (normals3d.go:11-79), normals/SJ (:82-185), Fscale (:188-207); arrays are (K, .)."""
    d = lambda D, F: F @ D.T  # (K,Np) rows: (D * F^T)^T
    xr, xs, xt = d(el.Dr, X), d(el.Ds, X), d(el.Dt, X)
    yr, ys, yt = d(el.Dr, Y), d(el.Ds, Y), d(el.Dt, Y)
    zr, zs, zt = d(el.Dr, Z), d(el.Ds, Z), d(el.Dt, Z)
    J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt)
    if np.any(J <= 0):
        raise ValueError("negative Jacobian")
    rx = (ys * zt - zs * yt) / J
    ry = -(xs * zt - zs * xt) / J
    rz = (xs * yt - ys * xt) / J
    sx = -(yr * zt - zr * yt) / J
    sy = (xr * zt - zr * xt) / J
    sz = -(xr * yt - yr * xt) / J
    tx = (yr * zs - zr * ys) / J
    ty = -(xr * zs - zr * xs) / J
    tz = (xr * ys - yr * xs) / J
    fm = el.Fmask
    parts = [(-tx[:, fm[0]], -ty[:, fm[0]], -tz[:, fm[0]]), (-sx[:, fm[1]], -sy[:, fm[1]], -sz[:, fm[1]]),
             (rx[:, fm[2]] + sx[:, fm[2]] + tx[:, fm[2]], ry[:, fm[2]] + sy[:, fm[2]] + ty[:, fm[2]],
              rz[:, fm[2]] + sz[:, fm[2]] + tz[:, fm[2]]),
             (-rx[:, fm[3]], -ry[:, fm[3]], -rz[:, fm[3]])]
    nx = np.concatenate([p[0] for p in parts], axis=1)
    ny = np.concatenate([p[1] for p in parts], axis=1)
    nz = np.concatenate([p[2] for p in parts], axis=1)
    mag = np.sqrt(nx * nx + ny * ny + nz * nz)
    if np.any(mag < 1e-14):
        raise ValueError("zero normal magnitude")
    nx, ny, nz = nx / mag, ny / mag, nz / mag
    Jf = J[:, fm.reshape(-1)]
    sJ = mag * Jf
    Fscale = sJ / Jf
    return Geometry(J, rx, ry, rz, sx, sy, sz, tx, ty, tz, nx, ny, nz, sJ, Fscale)


# --------------------------------------------------------------------------------------------------
# Connectivity: tiConnect3D and BuildMaps3D (+ the periodic variant this build specifies)
# --------------------------------------------------------------------------------------------------
FACE_VERTS = ((0, 1, 2), (0, 1, 3), (1, 2, 3), (0, 2, 3))  # ticonnect3d.go:41-46


def ti_connect3d(EToV):
    """Face matching by sorted vertex triple -> EToE, EToF (ticonnect3d.go:24-102)."""
    EToV = np.asarray(EToV, dtype=np.int64)
    K = EToV.shape[0]
    nn = int(EToV.max()) + 1
    fv = np.stack([np.sort(EToV[:, list(f)], axis=1) for f in FACE_VERTS], axis=1)  # (K,4,3)
    ids = (fv[..., 0] * nn * nn + fv[..., 1] * nn + fv[..., 2]).reshape(-1)
    order = np.argsort(ids, kind="stable")
    sid = ids[order]
    EToE = np.repeat(np.arange(K)[:, None], 4, axis=1)
    EToF = np.repeat(np.arange(4)[None, :], K, axis=0)
    eq = np.nonzero(sid[:-1] == sid[1:])[0]
    for i in eq:  # sequential like the reference: a later pair overwrites an earlier one
        a, b = order[i], order[i + 1]
        e1, f1, e2, f2 = a // 4, a % 4, b // 4, b % 4
        EToE[e1, f1], EToF[e1, f1] = e2, f2
        EToE[e2, f2], EToF[e2, f2] = e1, f1
    return EToE, EToF


def build_maps3d(el: RefElement, X, Y, Z, EToE, EToF, period=None, chunk=65536):
    """VmapM/VmapP/MapP by nearest face node within NODETOL (buildmaps3d.go:5-153), all face pairs at once in
    chunks of `chunk` faces.  Same arithmetic and the same first-minimum choice as the per-face loop
    (build_maps3d_loop, the line-by-line restatement), so the results are identical; this form scales to the
    benchmark meshes.

    ``period`` (a length-3 sequence or None) is this build's periodic extension: coordinate
    differences are wrapped into [-L/2, L/2] before the same NODETOL^2 distance test.
    """
    K, Np, Nfp = X.shape[0], el.Np, el.Nfp
    NF = Nfp * NFACES
    fm = el.Fmask.reshape(-1)
    vmapM = (fm[None, :] + (np.arange(K) * Np)[:, None]).reshape(-1)
    vmapP = vmapM.copy()
    mapP = np.arange(K * NF)
    x, y, z = X.reshape(-1), Y.reshape(-1), Z.reshape(-1)
    EToE = np.asarray(EToE, dtype=np.int64).reshape(-1)
    EToF = np.asarray(EToF, dtype=np.int64).reshape(-1)
    faces = np.arange(K * NFACES)
    k1, f1 = faces // NFACES, faces % NFACES
    conn = np.nonzero(~((EToE == k1) & (EToF == f1)))[0]  # faces with a neighbour (the loop skips the others)
    pts = np.arange(Nfp)

    def one(c0):
        fc = conn[c0:c0 + chunk]
        idsM = (fc // NFACES)[:, None] * NF + (fc % NFACES)[:, None] * Nfp + pts[None, :]
        idsP = EToE[fc][:, None] * NF + EToF[fc][:, None] * Nfp + pts[None, :]
        vidM, vidP = vmapM[idsM], vmapM[idsP]
        dx = x[vidP][:, None, :] - x[vidM][:, :, None]
        dy = y[vidP][:, None, :] - y[vidM][:, :, None]
        dz = z[vidP][:, None, :] - z[vidM][:, :, None]
        if period is not None:
            dx = _wrap(dx, period[0])
            dy = _wrap(dy, period[1])
            dz = _wrap(dz, period[2])
        D = dx * dx + dy * dy + dz * dz
        jmin = np.argmin(D, axis=2)
        ok = np.take_along_axis(D, jmin[..., None], axis=2)[..., 0] < NODETOL * NODETOL
        vmapP[idsM[ok]] = np.take_along_axis(vidP, jmin, axis=1)[ok]  # chunks write disjoint entries
        mapP[idsM[ok]] = np.take_along_axis(idsP, jmin, axis=1)[ok]

    parallel_chunks(one, len(conn), chunk)
    mapB = np.nonzero(mapP == np.arange(K * NF))[0]
    return vmapM, vmapP, mapP, mapB


def parallel_chunks(fn, n, chunk):
    """fn(c0) for c0 = 0, chunk, 2 chunk, ... < n on a thread pool (numpy releases the GIL in its kernels)."""
    starts = list(range(0, n, chunk))
    if len(starts) <= 1:
        return [fn(c0) for c0 in starts]
    with ThreadPoolExecutor(max_workers=min(len(starts), os.cpu_count() or 1)) as ex:
        return list(ex.map(fn, starts))


def build_maps3d_loop(el: RefElement, X, Y, Z, EToE, EToF, period=None):
    """Per-face loop form of build_maps3d, line by line after buildmaps3d.go:46-153 (checks the batched form)."""
    K, Np, Nfp = X.shape[0], el.Np, el.Nfp
    NF = Nfp * NFACES
    fm = el.Fmask.reshape(-1)
    vmapM = (fm[None, :] + (np.arange(K) * Np)[:, None]).reshape(-1)
    vmapP = vmapM.copy()
    mapP = np.arange(K * NF)
    x, y, z = X.reshape(-1), Y.reshape(-1), Z.reshape(-1)
    for k1 in range(K):
        for f1 in range(NFACES):
            k2, f2 = int(EToE[k1, f1]), int(EToF[k1, f1])
            if k2 == k1 and f2 == f1:
                continue
            idsM = k1 * NF + f1 * Nfp + np.arange(Nfp)
            idsP = k2 * NF + f2 * Nfp + np.arange(Nfp)
            vidM, vidP = vmapM[idsM], vmapM[idsP]
            dx = x[vidP][None, :] - x[vidM][:, None]
            dy = y[vidP][None, :] - y[vidM][:, None]
            dz = z[vidP][None, :] - z[vidM][:, None]
            if period is not None:
                dx = _wrap(dx, period[0])
                dy = _wrap(dy, period[1])
                dz = _wrap(dz, period[2])
            D = dx * dx + dy * dy + dz * dz
            jmin = np.argmin(D, axis=1)  # first minimum, as the strict '<' scan in the reference
            ok = D[np.arange(Nfp), jmin] < NODETOL * NODETOL
            vmapP[idsM[ok]] = vidP[jmin[ok]]
            mapP[idsM[ok]] = idsP[jmin[ok]]
    mapB = np.nonzero(mapP == np.arange(K * NF))[0]
    return vmapM, vmapP, mapP, mapB


def _wrap(d, L):
    """d - L where d > L/2, d + L where d < -L/2 (in place on a float array)."""
    d = np.array(d, dtype=np.float64, copy=True)
    np.subtract(d, L, out=d, where=d > 0.5 * L)
    np.add(d, L, out=d, where=d < -0.5 * L)
    return d


# --------------------------------------------------------------------------------------------------
# FaceConnector pick/place lists (utils/face_connector.go)
# --------------------------------------------------------------------------------------------------
@dataclass
class FaceConnector:
    nparts: int
    elems_per_part: list
    local_to_global: list
    pick: list = field(default_factory=list)   # pick[src][dst] -> np.int64 local source nodes
    place: list = field(default_factory=list)  # place[dst][src] -> np.int64 local P-buffer positions


def face_connector(K: int, Nfaces: int, Nfp: int, Np: int, vmapP, EToP) -> FaceConnector:
    """NewFaceConnector + BuildIndices (face_connector.go:43-187), one partition at a time: the destination
    partition's face points in (local element, point) order, split by source partition with a stable mask.
    That is the order in which the reference's per-element loop appends (face_connector_loop restates that
    loop), so the lists are identical."""
    vmapP = np.asarray(vmapP, dtype=np.int64)
    EToP = np.asarray(EToP, dtype=np.int64)
    if K <= 0 or Nfaces <= 0 or Nfp <= 0 or Np <= 0:
        raise ValueError("invalid dimensions")
    if len(vmapP) != K * Nfaces * Nfp or len(EToP) != K:
        raise ValueError("length mismatch")
    P = int(EToP.max()) + 1
    l2g = [np.nonzero(EToP == p)[0] for p in range(P)]
    g2l = np.zeros(K, dtype=np.int64)
    for p in range(P):
        g2l[l2g[p]] = np.arange(len(l2g[p]))
    NF = Nfaces * Nfp
    pick = [[None] * P for _ in range(P)]
    place = [[None] * P for _ in range(P)]
    for p in range(P):
        src = vmapP[(l2g[p][:, None] * NF + np.arange(NF)[None, :]).reshape(-1)]
        se = src // Np
        sp = EToP[se]
        lsrc = g2l[se] * Np + src % Np
        for q in range(P):
            sel = np.nonzero(sp == q)[0]
            pick[q][p] = lsrc[sel].astype(np.int64)
            place[p][q] = sel.astype(np.int64)  # = local element * NF + face point
    fc = FaceConnector(P, [len(v) for v in l2g], l2g)
    fc.pick, fc.place = pick, place
    return fc


def face_connector_loop(K: int, Nfaces: int, Nfp: int, Np: int, vmapP, EToP) -> FaceConnector:
    """Per-element loop form of face_connector after face_connector.go:143-187 (checks the batched form)."""
    vmapP = np.asarray(vmapP, dtype=np.int64)
    EToP = np.asarray(EToP, dtype=np.int64)
    if K <= 0 or Nfaces <= 0 or Nfp <= 0 or Np <= 0:
        raise ValueError("invalid dimensions")
    if len(vmapP) != K * Nfaces * Nfp or len(EToP) != K:
        raise ValueError("length mismatch")
    P = int(EToP.max()) + 1
    l2g = [np.nonzero(EToP == p)[0] for p in range(P)]
    g2l = np.zeros(K, dtype=np.int64)
    for p in range(P):
        g2l[l2g[p]] = np.arange(len(l2g[p]))
    pick = [[[] for _ in range(P)] for _ in range(P)]
    place = [[[] for _ in range(P)] for _ in range(P)]
    NF = Nfaces * Nfp
    for p in range(P):
        for le, ge in enumerate(l2g[p]):
            src = vmapP[ge * NF:(ge + 1) * NF]
            se = src // Np
            sp = EToP[se]
            lsrc = g2l[se] * Np + src % Np
            for q in np.unique(sp):
                sel = np.nonzero(sp == q)[0]
                pick[q][p].extend(lsrc[sel].tolist())
                place[p][q].extend((le * NF + sel).tolist())
    fc = FaceConnector(P, [len(v) for v in l2g], l2g)
    fc.pick = [[np.array(pick[a][b], dtype=np.int64) for b in range(P)] for a in range(P)]
    fc.place = [[np.array(place[a][b], dtype=np.int64) for b in range(P)] for a in range(P)]
    return fc


def face_connector_verify(fc: FaceConnector, Np: int, Nfaces: int, Nfp: int) -> None:
    """Index validity, pick/place length correspondence, conservation (face_connector.go:208-253)."""
    P = fc.nparts
    for p in range(P):
        for q in range(P):
            idx = fc.pick[p][q]
            if len(idx) and (idx.min() < 0 or idx.max() >= fc.elems_per_part[p] * Np):
                raise ValueError(f"invalid pick index for partition {p}")
            if len(fc.pick[p][q]) != len(fc.place[q][p]):
                raise ValueError("length mismatch")
    total = sum(len(fc.pick[p][q]) for p in range(P) for q in range(P))
    if total != sum(fc.elems_per_part) * Nfaces * Nfp:
        raise ValueError("conservation error")


def simulate_face_exchange(fc: FaceConnector, solutions, Nfaces: int, Nfp: int):
    """Pick -> exchange -> place into per-partition P buffers (utils/face_connector_test.go:98-157)."""
    P = fc.nparts
    pbufs = [np.zeros(fc.elems_per_part[p] * Nfaces * Nfp) for p in range(P)]
    for p in range(P):
        for q in range(P):
            pbufs[q][fc.place[q][p]] = np.asarray(solutions[p])[fc.pick[p][q]]
    return pbufs


# --------------------------------------------------------------------------------------------------
# Runner partition offsets (runner/builder/builder.go:113-159)
# --------------------------------------------------------------------------------------------------
def aligned_offsets(K, size_bytes: int, value_size: int, alignment: int):
    """Offsets in VALUES with per-partition byte alignment; returns (offsets, total_bytes)."""
    total = sum(K)
    bytes_per_elem = size_bytes // total
    vpe = bytes_per_elem // value_size
    alignment = alignment or 1
    off = []
    cur = 0
    for k in K:
        if cur % alignment:
            cur = ((cur + alignment - 1) // alignment) * alignment
        off.append(cur // value_size)
        cur += k * vpe * value_size
    if cur % alignment:
        cur = ((cur + alignment - 1) // alignment) * alignment
    off.append(cur // value_size)
    return off, off[-1] * value_size
