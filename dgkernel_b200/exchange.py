"""Slab exchange between ranks: the FaceConnector pick -> exchange -> place (utils/face_connector.go:143-187,
partitions/gather_scatter_array_design.md:176-228) with partitions spread over ranks, one rank per GPU.

Every rank holds its own x-slab partitions and, after them, a halo partition that receives the neighbour
values it reads from other ranks.  `halo_plan` (dgk_halo_plan) gives, per rank, the gather map of its face
points (remote neighbours pointing into the halo) and, per peer, the local values to send in wire order.  Per
stage: pack (dgk_gather_values into a send buffer), point-to-point send/receive with every peer that shares
faces (torch.distributed: NCCL between GPUs), unpack into the halo; then the rank's stage kernel runs with
halo=1 on its own partitions.  Nothing here reads another GPU's memory directly.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import mesh as M
from ._lib import check, lib
from .burgers import FACE, GEO, RK4A, RK4B, _TetBurgers, _pd, _pi
from .runner import Config, Float64, INT32, INT64, Input, Runner, Scalar, Temp

_PI64 = C.POINTER(C.c_int64)
_PI32 = C.POINTER(C.c_int32)


def _p(a, t):
    return a.ctypes.data_as(t)


def halo_plan(K, Nfp, Np, vmapP, EToP, part_rank, nranks, rank, local_off):
    """Exchange plan of `rank` (see dgk_halo_plan): dict with gmap (int32, the rank's face points partition by
    partition), send_idx (int64), send_count, recv_count, recv_off (per peer) and halo (values received)."""
    vmapP = np.ascontiguousarray(vmapP, dtype=np.int64).reshape(-1)
    EToP = np.ascontiguousarray(EToP, dtype=np.int64).reshape(-1)
    part_rank = np.ascontiguousarray(part_rank, dtype=np.int32)
    local_off = np.ascontiguousarray(local_off, dtype=np.int64)
    counts = np.zeros(3, dtype=np.int64)
    L = lib()
    args = (int(K), 4, int(Nfp), int(Np), _p(vmapP, _PI64), _p(EToP, _PI64), len(part_rank), _p(part_rank, _PI32),
            int(nranks), int(rank), _p(local_off, _PI64), _p(counts, _PI64))
    check(L.dgk_halo_plan(*args, None, None, None, None, None))
    gmap = np.zeros(int(counts[0]), dtype=np.int32)
    send_idx = np.zeros(max(int(counts[2]), 1), dtype=np.int64)
    sc, rc, ro = (np.zeros(nranks, dtype=np.int64) for _ in range(3))
    check(L.dgk_halo_plan(*args, _p(gmap, _PI32), _p(send_idx, _PI64), _p(sc, _PI64), _p(rc, _PI64), _p(ro, _PI64)))
    return {"gmap": gmap, "send_idx": send_idx[:int(counts[2])], "send_count": sc, "recv_count": rc, "recv_off": ro,
            "halo": int(counts[1])}


def slab_ranks(npart: int, nranks: int) -> np.ndarray:
    """Contiguous blocks of partitions per rank (x-slabs stay neighbours): rank of every partition."""
    if nranks < 1 or npart < nranks:
        raise ValueError("need at least one partition per rank")
    return np.array([p * nranks // npart for p in range(npart)], dtype=np.int32)


class BurgersSlab(_TetBurgers):
    """One rank's share of the plain FP64 Burgers stage on a periodic n^3 x 6 Kuhn mesh with nslab x-slab
    partitions spread over nranks ranks.  The global face matching `vmapP` (from one setup of the whole mesh)
    and the global time step `dt` are inputs; the rank allocates only its own slabs plus the halo.  `stream` (a
    torch.cuda.Stream) orders the stage, the pack and unpack kernels and the point-to-point transfers."""

    def __init__(self, N: int, n: int, nslab: int, nranks: int, rank: int, vmapP, dt: float, stream,
                 u0: str = "sine", conservative: int = 0):
        from .element import Element
        VX, VY, VZ, EToV, EToVp, EToP = M.kuhn_mesh(n, nslab)
        K = EToV.shape[0]
        el = Element(N)
        Np, Nfp = el.Np, el.Nfp
        part_rank = slab_ranks(nslab, nranks)
        Kp = K // nslab
        mine = [p for p in range(nslab) if part_rank[p] == rank]
        self.rank, self.nranks, self.part_rank, self.mine = rank, nranks, part_rank, mine
        # the plan needs the local value offsets; the runner's offsets follow from its partition sizes, so plan
        # once with provisional offsets to size the halo, then with the runner's own
        prov = np.concatenate(([0], np.cumsum([Kp * Np] * len(mine))))
        hp0 = halo_plan(K, Nfp, Np, vmapP, EToP, part_rank, nranks, rank, prov)
        kh = max(1, math.ceil(hp0["halo"] / Np))
        Kloc = [Kp] * len(mine) + [kh]
        elems = np.concatenate([np.arange(p * Kp, (p + 1) * Kp) for p in mine])
        EToVl = np.ascontiguousarray(np.concatenate((EToV[elems], np.repeat(EToV[:1], kh, axis=0))))
        Kt = EToVl.shape[0]
        selfE = np.repeat(np.arange(Kt, dtype=np.int64)[:, None], 4, axis=1)
        selfF = np.repeat(np.arange(4, dtype=np.int64)[None, :], Kt, axis=0)
        self.period = 0.0  # the gather map comes from the plan, not from a local face matching
        self.mixed = False
        self.tstream = stream
        self._assemble_local(N, el, VX, VY, VZ, EToVl, selfE, selfF, Kloc, stream.cuda_stream)
        r = self.runner
        off = r.GetOffsets("u")
        hp = halo_plan(K, Nfp, Np, vmapP, EToP, part_rank, nranks, rank, off[:len(mine) + 1])
        self.plan = hp
        NF = 4 * Nfp
        gm = np.zeros(Kt * NF, dtype=np.int32)
        gm[:len(hp["gmap"])] = hp["gmap"]
        r.CopyToDevice("gmap", gm)
        self.halo_off = int(off[len(mine)])
        kinds = {"sine": (0, 0.0, 0.5), "shock": (0, 0.5, 1.0), "smooth": (1, 0.5, 0.25)}
        kind, mean, amp = kinds[u0]
        check(lib().dgk_init_field(r._h, b"u", b"X", b"Y", b"Z", kind, mean, amp, 0, _pd(np.zeros(5))), r._h)
        self.conservative = conservative
        self.dt = dt
        self.stage = 0
        r.ConfigureKernel("rhsStage", *[r.Param(p) for p in ["u", "uNext", "resu", *GEO, *FACE, "gmap",
                                                              *self._fixed_m]],
                          r.Param("a"), r.Param("b"), r.Param("dt"))
        r.BuildKernel(f"rhsStage(conservative={conservative},halo=1)", "rhsStage")
        self.Kmine = Kp * len(mine)

    def _assemble_local(self, N, el, VX, VY, VZ, EToV, EToE, EToF, Kloc, stream):
        self.N, self.el, self.visc = N, el, None
        self.dtype = np.dtype(np.float64)
        Np, Nfp = el.Np, el.Nfp
        NF = 4 * Nfp
        K = self.K = EToV.shape[0]
        self.Kpart = list(Kloc)
        r = self.runner = Runner(Config(K=self.Kpart), stream=stream)
        sn = el.ShortName
        params = [Temp(nm).Type(Float64).Size(K * Np) for nm in ("u", "uNext", "resu", "X", "Y", "Z") + GEO]
        params += [Temp(nm).Type(Float64).Size(K * NF) for nm in FACE]
        params += [Temp("gmap").Type(INT32).Size(K * NF), Temp("vmapP").Type(INT64).Size(K * NF)]
        params += [Input(f"{m}_{sn}").Bind(getattr(el, m)).ToMatrix().Static() for m in ("Dr", "Ds", "Dt", "LIFT")]
        params += [Input("Fmask").Bind(el.Fmask.astype(np.float64)).ToMatrix().DeviceMemType(INT32)]
        params += [Scalar("a").Type(Float64), Scalar("b").Type(Float64), Scalar("dt").Type(Float64)]
        r.DefineBindings(*params)
        r.AllocateDevice()
        self._fixed_m = [f"Dr_{sn}", f"Ds_{sn}", f"Dt_{sn}", f"LIFT_{sn}", "Fmask"]
        names = ["X", "Y", "Z", *GEO, None, "nx", "ny", "nz", None, "Fscale", None, "vmapP"]
        carr = (C.c_char_p * 20)(*[None if v is None else v.encode() for v in names])
        hmin = C.c_double()
        check(lib().dgk_setup_geometry(r._h, el._h, len(VX), _pd(VX), _pd(VY), _pd(VZ), _pi(EToV), _pi(EToE),
                                       _pi(EToF), 0.0, carr, C.byref(hmin)), r._h)

    def own_state(self) -> np.ndarray:
        """The rank's own nodal values (its slabs, element-contiguous), without the halo."""
        return self.get("u")[:self.Kmine * self.el.Np]

    def pack(self, peer: int, dst_ptr: int):
        """Gather the values `peer` needs from the current state into the device buffer at dst_ptr."""
        hp = self.plan
        o = int(np.sum(hp["send_count"][:peer]))
        n = int(hp["send_count"][peer])
        if n == 0:
            return
        if not hasattr(self, "_send_idx_dev"):
            import torch
            self._send_idx_dev = torch.tensor(hp["send_idx"], dtype=torch.int64, device="cuda")
        idx_ptr = self._send_idx_dev.data_ptr() + 8 * o
        r = self.runner
        total = int(r.GetOffsets("u")[-1])
        check(lib().dgk_gather_values(C.c_void_p(r.DevicePtr("u")), Float64, total, C.c_void_p(idx_ptr), n,
                                      C.c_void_p(dst_ptr), C.c_void_p(self.tstream.cuda_stream)))

    def unpack(self, peer: int, src_ptr: int):
        """Place values received from `peer` (device buffer at src_ptr) into the halo of the current state."""
        hp = self.plan
        n = int(hp["recv_count"][peer])
        if n == 0:
            return
        import torch
        if not hasattr(self, "_iota") or self._iota.numel() < n:
            self._iota = torch.arange(max(n, 1), dtype=torch.int64, device="cuda")
        dst = self.runner.DevicePtr("u") + 8 * (self.halo_off + int(hp["recv_off"][peer]))
        check(lib().dgk_gather_values(C.c_void_p(src_ptr), Float64, n, C.c_void_p(self._iota.data_ptr()), n,
                                      C.c_void_p(dst), C.c_void_p(self.tstream.cuda_stream)))

    def exchange(self, group=None):
        """Pack -> send/receive with every peer sharing faces (torch.distributed, NCCL between GPUs) -> unpack
        into the halo, all ordered on the rank's stream.  Every rank calls this before each stage."""
        import torch
        import torch.distributed as dist
        hp = self.plan
        with torch.cuda.stream(self.tstream):
            reqs, bufs = [], []
            for q in range(self.nranks):
                if q == self.rank:
                    continue
                ns, nr = int(hp["send_count"][q]), int(hp["recv_count"][q])
                sb = torch.empty(max(ns, 1), dtype=torch.float64, device="cuda")
                rb = torch.empty(max(nr, 1), dtype=torch.float64, device="cuda")
                self.pack(q, sb.data_ptr())
                if ns:
                    reqs.append(dist.isend(sb[:ns], q, group=group))
                if nr:
                    reqs.append(dist.irecv(rb[:nr], q, group=group))
                bufs.append((q, sb, rb))
            for rq in reqs:
                rq.wait()
            for q, _, rb in bufs:
                self.unpack(q, rb.data_ptr())

    def run_stage(self):
        s = self.stage % 5
        self.runner.ExecuteKernel("rhsStage", RK4A[s], RK4B[s], self.dt)
        self.stage += 1
