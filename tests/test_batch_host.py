"""Host-side checks of the batching form (no GPU): seeded instance sizes, the side-by-side instance meshes
(every face connects inside its own instance, one partition per instance), and the autotuner's search and
cache logic with a stand-in measurement."""
import json
import os

import numpy as np

from dgkernel_b200 import autotune as T
from dgkernel_b200.burgers import _concat_meshes, ensemble_sizes
from oracle import burgers_ref as b


def test_ensemble_sizes_seeded_and_in_range():
    a = ensemble_sizes(256)
    assert a == ensemble_sizes(256)
    assert min(a) >= 6 and max(a) <= 24 and len(set(a)) > 10
    assert ensemble_sizes(16, seed=1) != ensemble_sizes(16, seed=2)
    # the splitmix64 stream of the oracle gives the same draw
    rng = b.SplitMix64(b.DEFAULT_SEED)
    assert a[:8] == [6 + int(np.floor(rng.uniform() * 19)) for _ in range(8)]


def test_instances_are_disjoint_partitions():
    sizes = [3, 4, 3, 5]  # n >= 3: with n = 2 the periodic wrap makes two faces of a cube identical
    VX, VY, VZ, EToV, EToE, EToF, EToP = _concat_meshes(sizes)
    K = [6 * n ** 3 for n in sizes]
    assert EToV.shape[0] == sum(K) and len(VX) == sum((n + 1) ** 3 for n in sizes)
    start = np.concatenate(([0], np.cumsum(K)))
    for i in range(len(sizes)):
        lo, hi = start[i], start[i + 1]
        assert np.all(EToP[lo:hi] == i)
        assert np.all((EToE[lo:hi] >= lo) & (EToE[lo:hi] < hi))  # periodic: every face inside the instance
        assert not np.any(EToE[lo:hi] == np.arange(lo, hi)[:, None])  # no boundary faces
        # reciprocity: the neighbour across face f points back through face EToF
        e = np.arange(lo, hi)[:, None].repeat(4, 1)
        assert np.all(EToE[EToE[lo:hi], EToF[lo:hi]] == e)


def test_autotune_search_and_cache(tmp_path):
    cands = [{"warps": 11, "ring": None}, {"warps": 8, "ring": 6}, {"warps": 4, "ring": None}]
    fake = {11: 1.0, 8: 0.7, 4: 1.4}
    best, times = T.search(cands, lambda c: fake[c["warps"]])
    assert best == {"warps": 8, "ring": 6} and len(times) == 3
    path = str(tmp_path / "sub" / "tune.json")
    key = T.problem_key("B200", "rhsStageMixed", 4, 55050240, 16)
    T.save_cache(path, {key: {"best": best, "ms_per_stage": times}})
    assert T.load_cache(path)[key]["best"] == best
    assert T.problem_key("B200", "rhsStageMixed", 4, 55050240 + 1000, 16) == key  # nearby sizes share
    assert T.problem_key("B200", "rhsStageMixed", 3, 55050240, 16) != key
    with open(path, "w") as f:
        f.write("not json")
    assert T.load_cache(path) == {}
    os.environ.pop("DGK_TUNE_CACHE", None)
    assert T.default_cache_path().endswith(os.path.join("dgkernel_b200", "tune.json"))


def test_autotune_candidates_by_order():
    """Orders 1..4 also try the tensor-core form of the mixed stage; order 5 has only the FP32-FMA form."""
    class P:
        def __init__(self, N):
            self.N = N
    c4, c5 = T.candidates_for(P(4)), T.candidates_for(P(5))
    assert any(c["mma"] for c in c4) and not any(c["mma"] for c in c5)
    assert all(c["warps"] in (8, 16) for c in c4 if c["mma"])
    assert c5 == T.MIXED_CANDIDATES
