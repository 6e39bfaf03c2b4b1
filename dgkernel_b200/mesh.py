"""Mesh-side setup from libdgk.so: periodic Kuhn-cube mesh, tiConnect3D, FaceConnector, gather map."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib

_PD = C.POINTER(C.c_double)
_PI64 = C.POINTER(C.c_int64)
_PI32 = C.POINTER(C.c_int32)


def _p(a, t):
    return a.ctypes.data_as(t)


def kuhn_mesh(n: int, nslab: int = 1, lo: float = -1.0, hi: float = 1.0):
    """n^3 cubes x 6 Kuhn tets on [lo,hi]^3, x-slab partitions.

    Returns VX, VY, VZ ((n+1)^3), EToV, EToV_periodic ((6n^3, 4)) and EToP (6n^3)."""
    nv, K = (n + 1) ** 3, 6 * n ** 3
    VX, VY, VZ = (np.zeros(nv) for _ in range(3))
    EToV = np.zeros((K, 4), dtype=np.int64)
    EToVp = np.zeros((K, 4), dtype=np.int64)
    EToP = np.zeros(K, dtype=np.int64)
    check(lib().dgk_kuhn_mesh(n, nslab, lo, hi, _p(VX, _PD), _p(VY, _PD), _p(VZ, _PD), _p(EToV, _PI64),
                              _p(EToVp, _PI64), _p(EToP, _PI64)))
    return VX, VY, VZ, EToV, EToVp, EToP


def read_gambit(path: str):
    """Gambit neutral file (tetrahedra) as read by ReadGambitNeutral (mesh/readers/gambit_reader.go:13-338):
    dict with VX, VY, VZ (vertices in file order), EToV [K, 4] (0-based), EToP [K] (partition N of the elements
    of group "p<N>", -1 unassigned) or None when the file has at most one element group, and bfaces [nb, 3]
    (element, 0-based Gambit face, boundary-set index)."""
    L = lib()
    counts = np.zeros(4, dtype=np.int64)
    p = str(path).encode()
    check(L.dgk_read_gambit(p, _p(counts, _PI64), None, None, None, None, None, None))
    nv, K, nb, parts = (int(v) for v in counts)
    VX, VY, VZ = np.zeros(nv), np.zeros(nv), np.zeros(nv)
    EToV = np.zeros((K, 4), dtype=np.int64)
    EToP = np.full(K, -1, dtype=np.int64)
    bf = np.zeros((nb, 3), dtype=np.int64)
    check(L.dgk_read_gambit(p, _p(counts, _PI64), _p(VX, _PD), _p(VY, _PD), _p(VZ, _PD), _p(EToV, _PI64),
                            _p(EToP, _PI64), _p(bf, _PI64) if nb else None))
    return {"VX": VX, "VY": VY, "VZ": VZ, "EToV": EToV, "EToP": EToP if parts else None, "bfaces": bf}


def ti_connect3d(EToV):
    """Element-to-element / element-to-face connectivity (gonudg ticonnect3d.go:24-102)."""
    EToV = np.ascontiguousarray(EToV, dtype=np.int64)
    K = EToV.shape[0]
    EToE = np.zeros((K, 4), dtype=np.int64)
    EToF = np.zeros((K, 4), dtype=np.int64)
    check(lib().dgk_ti_connect3d(K, _p(EToV, _PI64), _p(EToE, _PI64), _p(EToF, _PI64)))
    return EToE, EToF


class FaceConnector:
    """Pick/place lists per (source, target) partition pair (utils/face_connector.go)."""

    def __init__(self, K, Nfaces, Nfp, Np, vmapP, EToP):
        vmapP = np.ascontiguousarray(vmapP, dtype=np.int64).reshape(-1)
        EToP = np.ascontiguousarray(EToP, dtype=np.int64).reshape(-1)
        P = int(EToP.max()) + 1 if EToP.size else 0
        lens = np.zeros(P * P, dtype=np.int64)
        L = lib()
        check(L.dgk_face_connector(K, Nfaces, Nfp, Np, _p(vmapP, _PI64), _p(EToP, _PI64), P, _p(lens, _PI64), None,
                                   None))
        pick = np.zeros(int(lens.sum()), dtype=np.int64)
        place = np.zeros(int(lens.sum()), dtype=np.int64)
        check(L.dgk_face_connector(K, Nfaces, Nfp, Np, _p(vmapP, _PI64), _p(EToP, _PI64), P, _p(lens, _PI64),
                                   _p(pick, _PI64), _p(place, _PI64)))
        self.NumPartitions = P
        ptr = np.concatenate(([0], np.cumsum(lens)))
        # pick lists ordered by (src, dst); place lists by (dst, src)
        self.pick = [[pick[ptr[s * P + d]:ptr[s * P + d + 1]] for d in range(P)] for s in range(P)]
        place_lens = lens.reshape(P, P).T.reshape(-1)  # place[dst][src] has the length of pick[src][dst]
        pptr = np.concatenate(([0], np.cumsum(place_lens)))
        self.place = [[place[pptr[d * P + s]:pptr[d * P + s + 1]] for s in range(P)] for d in range(P)]
        self.ElemsPerPartition = [int(np.sum(EToP == p)) for p in range(P)]

    def GetPickIndices(self, src, dst):
        return self.pick[src][dst]

    def GetPlaceIndices(self, dst, src):
        return self.place[dst][src]


def face_gather_map(K, Nfaces, Nfp, Np, vmapP, EToP, node_off):
    """Absolute neighbour value index per face point, all partitions back to back (int32)."""
    vmapP = np.ascontiguousarray(vmapP, dtype=np.int64).reshape(-1)
    EToP = np.ascontiguousarray(EToP, dtype=np.int64).reshape(-1)
    node_off = np.ascontiguousarray(node_off, dtype=np.int64)
    gmap = np.zeros(K * Nfaces * Nfp, dtype=np.int32)
    check(lib().dgk_face_gather_map(K, Nfaces, Nfp, Np, _p(vmapP, _PI64), _p(EToP, _PI64), len(node_off) - 1,
                                    _p(node_off, _PI64), _p(gmap, _PI32)))
    return gmap


def compact_faces(Kpart, node_off, face_off, Np, Nfp, gmap):
    """Mixed-stage face connectivity from a gather map: (conn [slots, 5] int32, table [ncodes, Nfp] uint8)."""
    K = np.ascontiguousarray(Kpart, dtype=np.int64)
    slots = int(sum((k + 31) // 32 * 32 for k in K))
    conn = np.zeros(max(slots, 1) * 5, dtype=np.int32)
    table = np.zeros(256 * Nfp, dtype=np.uint8)
    nc = C.c_int32()
    g = np.ascontiguousarray(gmap, dtype=np.int32)
    no = np.ascontiguousarray(node_off, dtype=np.int64)
    fo = np.ascontiguousarray(face_off, dtype=np.int64)
    check(lib().dgk_compact_faces(len(K), _p(K, _PI64), _p(no, _PI64), _p(fo, _PI64), Np, Nfp, _p(g, _PI32),
                                  _p(conn, _PI32), table.ctypes.data_as(C.POINTER(C.c_uint8)), 256, C.byref(nc)))
    return conn[:slots * 5].reshape(slots, 5), table[:nc.value * Nfp].reshape(nc.value, Nfp)


def tile_halo(Kpart, node_off, Np, Nfp, conn, max_elems=128, max_halo=256, halo_floats=None, identity_code=255,
              align=4):
    """Tiles of the tensor-core mixed stage with their halos (dgk_tile_halo): dict with part, first, nelem,
    halo_off, halo_list ([entries, 2] int32) and tconn ([slots, 4] uint32)."""
    K = np.ascontiguousarray(Kpart, dtype=np.int64)
    no = np.ascontiguousarray(node_off, dtype=np.int64)
    cn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1)
    hf = max_elems * Np if halo_floats is None else halo_floats
    counts = np.zeros(2, dtype=np.int64)
    args = (len(K), _p(K, _PI64), _p(no, _PI64), Np, Nfp, _p(cn, _PI32), max_elems, max_halo, hf, identity_code,
            align, _p(counts, _PI64))
    check(lib().dgk_tile_halo(*args, None, None, None, None, None, None))
    nt, nh = int(counts[0]), int(counts[1])
    part, nelem, hoff = (np.zeros(nt + (i == 2), dtype=np.int32) for i in range(3))
    first = np.zeros(nt, dtype=np.int64)
    hl = np.zeros(max(2 * nh, 2), dtype=np.int32)
    tc = np.zeros(max(cn.size // 5 * 4, 4), dtype=np.uint32)
    check(lib().dgk_tile_halo(*args, _p(part, _PI32), _p(first, _PI64), _p(nelem, _PI32), _p(hoff, _PI32),
                              _p(hl, _PI32), tc.ctypes.data_as(C.POINTER(C.c_uint32))))
    return {"part": part, "first": first, "nelem": nelem, "halo_off": hoff, "halo_list": hl[:2 * nh].reshape(nh, 2),
            "tconn": tc[:cn.size // 5 * 4].reshape(-1, 4)}


def splitmix_uniform(seed: int, count: int) -> np.ndarray:
    out = np.zeros(count)
    check(lib().dgk_splitmix_uniform(seed, count, _p(out, _PD)))
    return out
