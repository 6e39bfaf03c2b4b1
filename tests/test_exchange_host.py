"""Slab exchange plan across ranks (dgk_halo_plan: the FaceConnector pick -> exchange -> place of
utils/face_connector.go:143-187 with partitions spread over ranks), on the host.

Each rank keeps its own x-slab partitions and a halo; its gather map reads remote neighbours from the halo,
which the peers fill with the values their send lists pick, in the wire order both sides derive from the pick
and place lists.  Bit-exact: every rank's face points must read exactly the values the single-rank gather
u[vmapP] reads, for 2 and 3 ranks in one process, and for 2 gloo ranks exchanging through torch.distributed.
"""
import os
import socket

import numpy as np
import pytest

from dgkernel_b200.exchange import halo_plan, slab_ranks
from oracle import burgers_ref as b


def _setup(N=2, n=6, nslab=6):
    ref = b.Problem(N, n, nslab, "sine")
    rng = np.random.default_rng(7)
    u = rng.standard_normal(ref.K * ref.el.Np)
    return ref, u


def _local(ref, u, part_rank, rank):
    Np = ref.el.Np
    Kp = ref.K // ref.nparts
    mine = [p for p in range(ref.nparts) if part_rank[p] == rank]
    off = np.arange(len(mine) + 1, dtype=np.int64) * Kp * Np
    own = np.concatenate([u[p * Kp * Np:(p + 1) * Kp * Np] for p in mine])
    face_pts = np.concatenate([np.arange(p * Kp * 4 * ref.el.Nfp, (p + 1) * Kp * 4 * ref.el.Nfp) for p in mine])
    return mine, off, own, face_pts


@pytest.mark.parametrize("W", [2, 3])
def test_halo_plan_reproduces_single_rank_gather(W):
    ref, u = _setup()
    part_rank = slab_ranks(ref.nparts, W)
    plans, owns, fps = [], [], []
    for r in range(W):
        mine, off, own, fp = _local(ref, u, part_rank, r)
        plans.append(halo_plan(ref.K, ref.el.Nfp, ref.el.Np, ref.vmapP, ref.EToP, part_rank, W, r, off))
        owns.append(own)
        fps.append(fp)
    for r in range(W):
        hp = plans[r]
        halo = np.zeros(hp["halo"])
        for q in range(W):
            if q == r:
                continue
            sq = plans[q]
            o = int(np.sum(sq["send_count"][:r]))
            vals = owns[q][sq["send_idx"][o:o + int(sq["send_count"][r])]]  # q packs for r
            assert len(vals) == hp["recv_count"][q]
            halo[hp["recv_off"][q]:hp["recv_off"][q] + len(vals)] = vals
        ext = np.concatenate((owns[r], halo))
        assert np.array_equal(ext[hp["gmap"]], u[np.asarray(ref.vmapP)[fps[r]]])
        # x-slabs: only the two neighbouring ranks exchange
        peers = [q for q in range(W) if q != r and hp["recv_count"][q] > 0]
        assert len(peers) == min(W - 1, 2)


def _gloo_rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ref, u = _setup()
        part_rank = slab_ranks(ref.nparts, world)
        mine, off, own, fp = _local(ref, u, part_rank, rank)
        hp = halo_plan(ref.K, ref.el.Nfp, ref.el.Np, ref.vmapP, ref.EToP, part_rank, world, rank, off)
        halo = np.zeros(hp["halo"])
        reqs, recv = [], []
        for q in range(world):
            if q == rank:
                continue
            o = int(np.sum(hp["send_count"][:q]))
            send = torch.tensor(own[hp["send_idx"][o:o + int(hp["send_count"][q])]])
            rb = torch.empty(int(hp["recv_count"][q]), dtype=torch.float64)
            reqs += [dist.isend(send, q), dist.irecv(rb, q)]
            recv.append((q, rb))
        for rq in reqs:
            rq.wait()
        for q, rb in recv:
            halo[hp["recv_off"][q]:hp["recv_off"][q] + rb.numel()] = rb.numpy()
        ext = np.concatenate((own, halo))
        ok = bool(np.array_equal(ext[hp["gmap"]], u[np.asarray(ref.vmapP)[fp]]))
        out.put((rank, ok))
    finally:
        dist.destroy_process_group()


def test_halo_exchange_over_two_gloo_ranks():
    import multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: True, 1: True}
