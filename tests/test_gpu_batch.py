"""Batching form on the GPU: independent instances of uneven size advanced by one stage launch, the stage
sequence replayed from a captured CUDA graph, and the launch-shape autotuner.

Bounds: each instance against the FP64 oracle run of that instance alone (same u0, the batch's common dt),
relative L2 <= MIXED_TOL = 1e-7 after 10 stages; graph replay and tuned launch shapes against plain
ExecuteKernel launches: bit-identical (the same per-element arithmetic runs in every case).
"""
import numpy as np
import pytest

from dgkernel_b200 import autotune as T
from dgkernel_b200.burgers import BurgersEnsemble, MIXED
from oracle import burgers_ref as b
from oracle import oracle as O

from conftest import rel_l2

pytestmark = pytest.mark.gpu
MIXED_TOL = 1e-7
SIZES = [3, 4, 3, 5]


def test_instances_match_their_own_oracle_runs():
    E = BurgersEnsemble(3, SIZES)
    u0 = E.u0.copy()
    E.run_stages(10)
    u = E.get("u")
    for i, n in enumerate(SIZES):
        ref = b.Problem(3, n, 1, "sine")
        ui = np.ascontiguousarray(E.instance(i, u0)).copy()
        resu = np.zeros_like(ui)
        O.RunState(ref).run(ui, resu, E.dt, 10, threads=4)
        err = rel_l2(E.instance(i, u), ui)
        assert err < MIXED_TOL, (i, err)
    E.free()


def test_instance_initial_fields_follow_their_seeds():
    E = BurgersEnsemble(3, SIZES)
    for i, n in enumerate(SIZES):
        ref = b.Problem(3, n, 1, "sine")
        want = b.u0_modes(ref.X, ref.Y, ref.Z, b.random_modes(b.SplitMix64(b.DEFAULT_SEED + i)))
        assert rel_l2(E.instance(i, E.u0), want) < 1e-14
    E.free()


def test_graph_replay_matches_launches():
    A = BurgersEnsemble(3, SIZES)
    B = BurgersEnsemble(3, SIZES)
    A.run_stages(20)
    g = B.capture_steps(2)
    B.run_graph(g, 2)
    assert np.array_equal(A.get("u"), B.get("u"))
    g.Free()
    A.free()
    B.free()


def test_autotune_keeps_state_and_results(tmp_path):
    A = BurgersEnsemble(3, SIZES)
    B = BurgersEnsemble(3, SIZES)
    before = B.get("u")
    best = T.autotune(B, cache_path=str(tmp_path / "tune.json"), stages=2)
    assert best in T.candidates_for(B)
    assert np.array_equal(B.get("u"), before)  # tuning stages run with dt = 0
    A.build_stage(**best)  # the same form and launch shape: the same bits
    A.run_stages(10)
    B.run_stages(10)
    assert np.array_equal(A.get("u"), B.get("u"))
    again = T.autotune(B, cache_path=str(tmp_path / "tune.json"))  # from the cache
    assert again == best
    A.free()
    B.free()
