"""Slab exchange on the GPU, two ranks emulated in one process on one device: each rank's problem
(BurgersSlab: its own x-slabs plus a halo, the plain FP64 stage with halo=1) packs the values its peer needs
with the library's gather kernel, the peer unpacks them into its halo, and both advance.  Ten LSERK4 stages
must reproduce the single-rank stage bit for bit (the same per-element arithmetic reads the same values).
The transfers between the two problems stand in for the NCCL send/receive of a two-GPU run."""
import numpy as np
import pytest
import torch

from dgkernel_b200.burgers import BurgersProblem
from dgkernel_b200.exchange import BurgersSlab

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,n,nslab,W", [(2, 4, 4, 2), (4, 6, 6, 3)])
def test_two_rank_slab_exchange_matches_single_rank(N, n, nslab, W):
    st = torch.cuda.Stream()
    G = BurgersProblem(N, n, nslab, np.float64, "sine", stream=st.cuda_stream)
    ranks = [BurgersSlab(N, n, nslab, W, r, G.vmapP, G.dt, st) for r in range(W)]
    for s in range(10):
        for r in range(W):
            for q in range(W):
                cnt = int(ranks[q].plan["send_count"][r])
                if q == r or cnt == 0:
                    continue
                buf = torch.empty(cnt, dtype=torch.float64, device="cuda")
                with torch.cuda.stream(st):
                    ranks[q].pack(r, buf.data_ptr())
                    ranks[r].unpack(q, buf.data_ptr())
                st.synchronize()
        for R in ranks:
            R.run_stage()
    G.run_stages(10)
    want = G.get("u")
    got = np.concatenate([R.own_state() for R in ranks])
    assert np.array_equal(got, want), float(np.max(np.abs(got - want)))
    for R in ranks:
        R.free()
    G.free()
