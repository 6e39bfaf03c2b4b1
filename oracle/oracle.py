"""ctypes front end of the CPU oracle (test infrastructure only).

Loads oracle/_build/libdgk_oracle.so (built by oracle/Makefile) and exposes numpy-friendly wrappers of
the restated OKL kernels.  Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libdgk_oracle.so")
_lib = None

_d = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.ora_matmul.argtypes = [_d, C.c_int, C.c_int, C.c_int, _i64, _d, _i64, _d, _i64, C.c_int]
        L.ora_differentiate.argtypes = [C.c_int, _d, _d, _d, C.c_int, _i64, _i64] + [_d] * 16 + [C.c_int]
        L.ora_compute_rhs_volume.argtypes = [C.c_int, _d, _d, _d, C.c_int, _i64, _i64] + [_d] * 14 + [C.c_int]
        L.ora_update_ref.argtypes = [C.c_int, C.c_int, _i64, _i64, _d, _d, _d, C.c_double, C.c_double]
        L.ora_exchange.argtypes = [C.c_int, _d, _i64, _i64, _i64, _i64, _i64, _d, _i64]
        L.ora_rhs_lf.argtypes = ([C.c_int, C.c_int, _d, _d, _d, _d, _i32, C.c_int, _i64, _i64, _i64] + [_d] * 14
                                 + [_i64] * 4 + [_d, _d, C.c_int, C.c_int])
        L.ora_run.argtypes = ([C.c_int, C.c_int, _d, _d, _d, _d, _i32, C.c_int, _i64, _i64, _i64] + [_d] * 15
                              + [_i64] * 4 + [C.c_double, C.c_int, C.c_long, C.c_int, C.c_int])
        L.ora_run.restype = C.c_long
        L.ora_lserk_coefficients.argtypes = [_d, _d]
        L.ora_mlp_forward1.argtypes = [C.c_int, _d, _d]
        L.ora_mlp_forward1.restype = C.c_double
        L.ora_sensor.argtypes = [C.c_int, _d, _i32, C.c_long, _d, C.c_double, C.c_double, _d, _d, C.c_void_p]
        av_common = ([C.c_int, C.c_int, C.c_int, _d, _d, _d, _d, _d, _i32, _i32, C.c_long, _d] + [_d] * 13 +
                     [_i64, C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_double, C.c_double])
        L.ora_rhs_av.argtypes = av_common[:11] + [_d] + av_common[12:] + [_d, C.c_void_p, C.c_int]
        L.ora_run_av.argtypes = (av_common[:11] + [_d, _d] + av_common[12:] +
                                 [C.c_double, C.c_int, C.c_long, C.c_int])
        L.ora_run_av.restype = C.c_long
        L.ora_max_threads.restype = C.c_int
        _lib = L
    return _lib


def cm(M) -> np.ndarray:
    """Column-major copy of a row-major matrix (the device/static matrix layout, builder.go:251-252, 378)."""
    return np.ascontiguousarray(np.asarray(M, dtype=np.float64).T).reshape(-1)


def lserk_coefficients():
    a, b = np.zeros(5), np.zeros(5)
    lib().ora_lserk_coefficients(a, b)
    return a, b


def max_threads() -> int:
    return int(lib().ora_max_threads())


def csr_pairs(lists, nparts):
    """Flatten lists[a][b] (numpy int arrays) into (ptr, idx) over pairs a*nparts+b."""
    ptr = np.zeros(nparts * nparts + 1, dtype=np.int64)
    chunks = []
    for a in range(nparts):
        for b in range(nparts):
            arr = np.asarray(lists[a][b], dtype=np.int64)
            ptr[a * nparts + b + 1] = ptr[a * nparts + b] + len(arr)
            chunks.append(arr)
    idx = np.concatenate(chunks) if chunks else np.zeros(0, np.int64)
    return ptr, np.ascontiguousarray(idx, dtype=np.int64)


def _flat(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))


def _offsets(K, per_elem):
    off = np.zeros(len(K) + 1, dtype=np.int64)
    off[1:] = np.cumsum(np.asarray(K, dtype=np.int64) * per_elem)
    return off


def differentiate(el, K, U, geo_arrays, threads=1):
    """Volume derivative microbench on contiguous partitions; returns (DuDx, DuDy, DuDz) flat."""
    Np = el.Np
    off = _offsets(K, Np)
    U = _flat(U)
    g = [_flat(a) for a in geo_arrays]
    tmp = [np.zeros_like(U) for _ in range(6)]
    lib().ora_differentiate(Np, cm(el.Dr), cm(el.Ds), cm(el.Dt), len(K), np.asarray(K, np.int64), off, U, *g,
                            *tmp, threads)
    return tmp[3], tmp[4], tmp[5]


class RunState:
    """Packed arrays for ora_rhs_lf / ora_run built from an oracle Problem (contiguous partitions)."""

    def __init__(self, prob):
        el, geo = prob.el, prob.geo
        self.prob = prob
        self.Np, self.Nfp = el.Np, el.Nfp
        self.K = np.asarray(prob.Kpart, dtype=np.int64)
        self.noff = _offsets(self.K, el.Np)
        self.foff = _offsets(self.K, 4 * el.Nfp)
        self.mats = [cm(el.Dr), cm(el.Ds), cm(el.Dt), cm(el.LIFT)]
        self.fmask = np.ascontiguousarray(el.Fmask.reshape(-1).astype(np.int32))
        self.geo = [_flat(getattr(geo, n)) for n in ("rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz")]
        self.face = [_flat(getattr(geo, n)) for n in ("nx", "ny", "nz", "Fscale")]
        P = prob.fc.nparts
        self.pick_ptr, self.pick_idx = csr_pairs(prob.fc.pick, P)
        self.place_ptr, self.place_idx = csr_pairs(prob.fc.place, P)

    def rhs(self, u, conservative=0, threads=1):
        u = _flat(u)
        pbuf = np.zeros(int(self.foff[-1]))
        rhs = np.zeros(int(self.noff[-1]))
        lib().ora_rhs_lf(self.Np, self.Nfp, *self.mats, self.fmask, len(self.K), self.K, self.noff, self.foff, u,
                         *self.geo, *self.face, self.pick_ptr, self.pick_idx, self.place_ptr, self.place_idx, pbuf,
                         rhs, conservative, threads)
        return rhs

    def run(self, u, resu, dt, nstages, stage0=0, conservative=0, threads=1):
        """Advance (u, resu) in place by `nstages` LSERK4 stages starting at stage index `stage0`."""
        assert u.dtype == np.float64 and u.flags.c_contiguous and resu.flags.c_contiguous
        return lib().ora_run(self.Np, self.Nfp, *self.mats, self.fmask, len(self.K), self.K, self.noff, self.foff,
                             u.reshape(-1), resu.reshape(-1), *self.geo, *self.face, self.pick_ptr, self.pick_idx,
                             self.place_ptr, self.place_idx, float(dt), int(stage0), int(nstages), conservative,
                             threads)


def mode_degrees(N):
    """Total degree of every orthonormal mode, modes ordered i, j, k (vandermonde3d.go:15-42)."""
    return np.array([i + j + k for i in range(N + 1) for j in range(N - i + 1) for k in range(N - i - j + 1)])


class AVState:
    """Artificial-viscosity oracle on one packed mesh (all partitions contiguous; neighbour traces through
    the global VmapP)."""

    MODES = {"none": 0, "pp": 1, "mlp": 2, "mlp0": 3}  # mlp0: network outputs <= lo are smooth (eps = 0)

    def __init__(self, prob, eps0=1.0, c0=0.0, kappa=1.0, conf=(0.1, 0.9)):
        el, geo = prob.el, prob.geo
        self.prob, self.N, self.Np, self.Nfp, self.K = prob, prob.N, el.Np, el.Nfp, prob.K
        self.mats = [cm(el.Dr), cm(el.Ds), cm(el.Dt), cm(el.LIFT)]
        self.vinv = cm(el.Vinv)
        self.top = np.ascontiguousarray((mode_degrees(prob.N) == prob.N).astype(np.int32))
        self.fmask = np.ascontiguousarray(el.Fmask.reshape(-1).astype(np.int32))
        self.geo = [_flat(getattr(geo, n)) for n in ("rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz")]
        self.face = [_flat(getattr(geo, n)) for n in ("nx", "ny", "nz", "Fscale")]
        self.vmapP = np.ascontiguousarray(np.asarray(prob.vmapP, dtype=np.int64).reshape(-1))
        self.eps0, self.kappa, self.conf = float(eps0), float(kappa), conf
        self.s0 = -(float(c0) + 4.0 * np.log10(prob.N))

    def _mlp(self, mlp):
        if mlp is None:
            return None
        return np.ascontiguousarray(np.asarray(mlp, dtype=np.float64))

    def sensor(self, u):
        u = _flat(u)
        S = np.zeros(self.K)
        sig = np.zeros(self.K)
        feat = np.zeros(self.K * self.Np)
        lib().ora_sensor(self.Np, self.vinv, self.top, self.K, u, self.s0, self.kappa, S, sig,
                         feat.ctypes.data_as(C.c_void_p))
        return S, sig, feat.reshape(self.K, self.Np)

    def rhs(self, u, mode="pp", mlp=None, threads=4):
        u = _flat(u)
        out = np.zeros_like(u)
        eps = np.zeros(self.K)
        m = self._mlp(mlp)
        lib().ora_rhs_av(self.Np, self.Nfp, self.N, *self.mats, self.vinv, self.top, self.fmask, self.K, u,
                         *self.geo, *self.face, self.vmapP, self.MODES[mode], self.eps0, self.s0, self.kappa,
                         None if m is None else m.ctypes.data_as(C.c_void_p), self.conf[0], self.conf[1], out,
                         eps.ctypes.data_as(C.c_void_p), threads)
        return out, eps

    def run(self, u, resu, dt, nstages, mode="pp", mlp=None, stage0=0, threads=4):
        m = self._mlp(mlp)
        return lib().ora_run_av(self.Np, self.Nfp, self.N, *self.mats, self.vinv, self.top, self.fmask, self.K,
                                u.reshape(-1), resu.reshape(-1), *self.geo, *self.face, self.vmapP,
                                self.MODES[mode], self.eps0, self.s0, self.kappa,
                                None if m is None else m.ctypes.data_as(C.c_void_p), self.conf[0], self.conf[1],
                                float(dt), int(stage0), int(nstages), threads)
