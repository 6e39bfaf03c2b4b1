"""Oracle-side problem setup for the 3-D scalar Burgers tet-DG benchmarks (test infrastructure only).

The reference ships no periodic structured mesh, seeded initial conditions or shock-time estimate; this
module restates the formulas the build fixes for them (the product implements the same formulas in
C++ and is checked against this file):

  * splitmix64 -> uniform doubles (53-bit), Box-Muller normals from two uniforms (cosine branch);
  * an n^3 cube grid on [-1,1]^3, each cube cut into 6 Kuhn tets along (0,0,0)->(1,1,1) in the tet
    order and orientation of utils/mesh_test_helpers.go:346-388, cubes numbered x-slowest so that
    x-slab partitions are contiguous element ranges;
  * periodic faces via wrapped vertex ids in tiConnect3D and coordinates compared modulo 2;
  * dt = CFL * h_min / max|u0|, h_min the smallest node-pair distance in any element
    (examples/3d_scalar_burgers_equation.go:415-428, 697-717).
"""
from __future__ import annotations

import math

import numpy as np

from . import gonudg_ref as g

MASK64 = (1 << 64) - 1
DEFAULT_SEED = 20261203


class SplitMix64:
    """splitmix64 stream; uniform() = (z >> 11) * 2^-53 in [0, 1)."""

    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / 9007199254740992.0)

    def normal(self) -> float:
        u1 = 1.0 - self.uniform()  # (0, 1]
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


# Kuhn split of the unit cube: corner bits (x, y, z); tet order of utils/mesh_test_helpers.go:353-366.
_CORNER = {"o": (0, 0, 0), "x": (1, 0, 0), "y": (0, 1, 0), "z": (0, 0, 1), "xy": (1, 1, 0), "xz": (1, 0, 1),
           "yz": (0, 1, 1), "xyz": (1, 1, 1)}
KUHN_TETS = (("o", "x", "xy", "xyz"), ("o", "xy", "y", "xyz"), ("o", "z", "xz", "xyz"),
             ("o", "yz", "z", "xyz"), ("o", "xz", "x", "xyz"), ("o", "y", "yz", "xyz"))


def kuhn_mesh(n: int, nparts: int = 1, lo: float = -1.0, hi: float = 1.0):
    """Return VX, VY, VZ, EToV (geometric ids), EToV_per (wrapped ids for periodic matching), EToP."""
    if n < 2:
        raise ValueError("periodic Kuhn mesh needs n >= 2")
    if n % nparts:
        raise ValueError("n must be divisible by the number of x-slabs")
    h = (hi - lo) / n
    m = n + 1
    ii, jj, kk = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    VX = (lo + h * ii).reshape(-1).astype(np.float64)
    VY = (lo + h * jj).reshape(-1).astype(np.float64)
    VZ = (lo + h * kk).reshape(-1).astype(np.float64)
    ci, cj, ck = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ci, cj, ck = ci.reshape(-1), cj.reshape(-1), ck.reshape(-1)  # cube c = (i*n + j)*n + k
    EToV = np.zeros((n ** 3 * 6, 4), dtype=np.int64)
    EToVp = np.zeros_like(EToV)
    for t, tet in enumerate(KUHN_TETS):
        for v, name in enumerate(tet):
            dx, dy, dz = _CORNER[name]
            gi, gj, gk = ci + dx, cj + dy, ck + dz
            EToV[t::6, v] = (gi * m + gj) * m + gk
            EToVp[t::6, v] = ((gi % n) * n + (gj % n)) * n + (gk % n)
    EToP = np.repeat(ci // (n // nparts), 6).astype(np.int64)
    return VX, VY, VZ, EToV, EToVp, EToP


def u0_sine(X, Y, Z, amp=0.5, offset=0.0):
    """u0 = offset + amp sin(pi x) sin(pi y) sin(pi z)."""
    return offset + amp * np.sin(np.pi * X) * np.sin(np.pi * Y) * np.sin(np.pi * Z)


def u0_smooth_c3(X, Y, Z):
    """u0 = 0.5 + 0.25 sin(pi x) cos(pi y) sin(pi z)."""
    return 0.5 + 0.25 * np.sin(np.pi * X) * np.cos(np.pi * Y) * np.sin(np.pi * Z)


def random_modes(rng: SplitMix64, nmodes: int = 8, kmax: int = 3, sigma: float = 0.1):
    """Modes (k, a, phi): k integer in [-kmax,kmax]^3 with 0 < |k| <= kmax by rejection, a ~ N(0, sigma^2),
    phi ~ U[0, 2pi)."""
    modes = []
    for _ in range(nmodes):
        while True:
            k = [int(math.floor(rng.uniform() * (2 * kmax + 1))) - kmax for _ in range(3)]
            k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2]
            if 0 < k2 <= kmax * kmax:
                break
        a = sigma * rng.normal()
        phi = 2.0 * math.pi * rng.uniform()
        modes.append((k, a, phi))
    return modes


def u0_modes(X, Y, Z, modes, mean: float = 0.5):
    u = np.full(np.shape(X), mean)
    for k, a, phi in modes:
        u = u + a * np.cos(np.pi * (k[0] * X + k[1] * Y + k[2] * Z) + phi)
    return u


def h_min(X, Y, Z, chunk=8192) -> float:
    """Smallest node-pair distance > 1e-12 over all elements (3d_scalar_burgers_equation.go:697-717), in chunks
    of elements; the same distances as the per-element loop (h_min_loop), so the same minimum."""
    K, Np = X.shape
    iu = np.triu_indices(Np, 1)

    def one(c0):
        x, y, z = X[c0:c0 + chunk], Y[c0:c0 + chunk], Z[c0:c0 + chunk]
        dx = x[:, :, None] - x[:, None, :]
        dy = y[:, :, None] - y[:, None, :]
        dz = z[:, :, None] - z[:, None, :]
        d = np.sqrt(dx * dx + dy * dy + dz * dz)[:, iu[0], iu[1]]
        d = d[d > 1e-12]
        return float(d.min()) if d.size else math.inf

    return min(g.parallel_chunks(one, K, chunk), default=math.inf)


def h_min_loop(X, Y, Z) -> float:
    """Per-element loop form of h_min (checks the chunked form)."""
    best = math.inf
    for k in range(X.shape[0]):
        p = np.stack((X[k], Y[k], Z[k]), axis=1)
        d = np.sqrt(np.sum((p[:, None, :] - p[None, :, :]) ** 2, axis=2))
        d = d[np.triu_indices(len(p), 1)]
        d = d[d > 1e-12]
        best = min(best, float(d.min()))
    return best


class Problem:
    """All arrays one configuration binds, element-contiguous (K, Np) / (K, 4 Nfp)."""

    def __init__(self, N: int, n: int, nparts: int, u0: str = "sine", seed: int = DEFAULT_SEED, cfl: float = 0.3):
        self.N, self.n, self.nparts = N, n, nparts
        self.el = g.ref_element(N)
        VX, VY, VZ, EToV, EToVp, EToP = kuhn_mesh(n, nparts)
        self.VX, self.VY, self.VZ, self.EToV, self.EToVp, self.EToP = VX, VY, VZ, EToV, EToVp, EToP
        self.K = EToV.shape[0]
        self.X, self.Y, self.Z = g.node_coords(self.el, VX, VY, VZ, EToV)
        self.geo = g.geometric_factors(self.el, self.X, self.Y, self.Z)
        self.EToE, self.EToF = g.ti_connect3d(EToVp)
        self.vmapM, self.vmapP, self.mapP, self.mapB = g.build_maps3d(self.el, self.X, self.Y, self.Z, self.EToE,
                                                                      self.EToF, period=(2.0, 2.0, 2.0))
        self.fc = g.face_connector(self.K, 4, self.el.Nfp, self.el.Np, self.vmapP, EToP)
        self.Kpart = [int(v) for v in self.fc.elems_per_part]
        if u0 == "sine":
            self.u0 = u0_sine(self.X, self.Y, self.Z)
        elif u0 == "shock":
            self.u0 = u0_sine(self.X, self.Y, self.Z, amp=1.0, offset=0.5)
        elif u0 == "smooth":
            self.u0 = u0_smooth_c3(self.X, self.Y, self.Z)
        elif u0 == "modes":
            self.u0 = u0_modes(self.X, self.Y, self.Z, random_modes(SplitMix64(seed)))
        else:
            raise ValueError(u0)
        self.hmin = h_min(self.X, self.Y, self.Z)
        self.dt = cfl * self.hmin / float(np.max(np.abs(self.u0)))


class MeshProblem(Problem):
    """The arrays of a Burgers problem on an unstructured tetrahedral mesh (not periodic: unmatched faces keep
    VmapP = VmapM, buildmaps3d.go:34), elements stored partition by partition in ascending partition id, then
    ascending element id (the FaceConnector's local numbering), partitions renumbered 0.. in that order."""

    def __init__(self, N: int, VX, VY, VZ, EToV, EToP=None, u0: str = "sine", cfl: float = 0.3):
        EToV = np.asarray(EToV, dtype=np.int64)
        K = EToV.shape[0]
        EToP = np.zeros(K, dtype=np.int64) if EToP is None else np.asarray(EToP, dtype=np.int64)
        order = np.argsort(EToP, kind="stable")
        ids, counts = np.unique(EToP, return_counts=True)
        self.N, self.n, self.nparts = N, 0, len(ids)
        self.el = g.ref_element(N)
        self.VX, self.VY, self.VZ = (np.asarray(v, dtype=np.float64) for v in (VX, VY, VZ))
        self.EToV = EToV[order]
        self.EToP = np.repeat(np.arange(len(ids), dtype=np.int64), counts)
        self.order = order
        self.K = K
        self.X, self.Y, self.Z = g.node_coords(self.el, self.VX, self.VY, self.VZ, self.EToV)
        self.geo = g.geometric_factors(self.el, self.X, self.Y, self.Z)
        self.EToE, self.EToF = g.ti_connect3d(self.EToV)
        self.vmapM, self.vmapP, self.mapP, self.mapB = g.build_maps3d(self.el, self.X, self.Y, self.Z, self.EToE,
                                                                      self.EToF, period=None)
        self.fc = g.face_connector(self.K, 4, self.el.Nfp, self.el.Np, self.vmapP, self.EToP)
        self.Kpart = [int(v) for v in self.fc.elems_per_part]
        if u0 == "sine":
            self.u0 = u0_sine(self.X, self.Y, self.Z)
        elif u0 == "shock":
            self.u0 = u0_sine(self.X, self.Y, self.Z, amp=1.0, offset=0.5)
        elif u0 == "smooth":
            self.u0 = u0_smooth_c3(self.X, self.Y, self.Z)
        else:
            raise ValueError(u0)
        self.hmin = h_min(self.X, self.Y, self.Z)
        self.dt = cfl * self.hmin / float(np.max(np.abs(self.u0)))
