"""Reference tetrahedron operators (gonudg's NewDG3D mesh-independent half) from libdgk.so."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib


class Element:
    """Order-N nodal tetrahedron: nodes r,s,t, V, Vinv, MassMatrix, M, Minv, Dr, Ds, Dt, LIFT, Fmask.

    Matrices are row-major numpy arrays, named as GetRefMatrices (tetnudg/tet_nudg_mesh.go:371-389)."""

    def __init__(self, N: int):
        L = lib()
        h = C.c_void_p()
        check(L.dgk_element_create(int(N), C.byref(h)))
        self._h = h
        np_, nfp = C.c_int32(), C.c_int32()
        check(L.dgk_element_dims(h, C.byref(np_), C.byref(nfp)))
        self.N, self.Np, self.Nfp = int(N), np_.value, nfp.value
        self.NFaces = 4
        for name in ("r", "s", "t"):
            setattr(self, name, self._get(name, (self.Np,)))
        for name in ("V", "Vinv", "MassMatrix", "M", "Minv", "Dr", "Ds", "Dt"):
            setattr(self, name, self._get(name, (self.Np, self.Np)))
        self.LIFT = self._get("LIFT", (self.Np, 4 * self.Nfp))
        fm = np.zeros(4 * self.Nfp, dtype=np.int32)
        check(L.dgk_element_fmask(h, fm.ctypes.data_as(C.POINTER(C.c_int32))))
        self.Fmask = fm.reshape(4, self.Nfp)

    def _get(self, what, shape):
        out = np.zeros(shape, dtype=np.float64)
        check(lib().dgk_element_get(self._h, what.encode(), out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
        return out

    @property
    def ShortName(self) -> str:
        return f"NudgTet{self.N}"

    def ref_matrices(self) -> dict:
        sn = self.ShortName
        return {f"V_{sn}": self.V, f"Vinv_{sn}": self.Vinv, f"M_{sn}": self.M, f"Minv_{sn}": self.Minv,
                f"Dr_{sn}": self.Dr, f"Ds_{sn}": self.Ds, f"Dt_{sn}": self.Dt, f"LIFT_{sn}": self.LIFT}

    def __del__(self):
        try:
            if self._h:
                lib().dgk_element_free(self._h)
                self._h = None
        except Exception:
            pass
