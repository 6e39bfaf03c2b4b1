"""Launch-shape autotuner for the stage operators.

For a built problem (`BurgersProblem` or `BurgersEnsemble`) the tuner rebuilds the stage operator with each
candidate launch shape, times a few stages of it (host clock between two stream synchronisations), keeps the fastest
and caches the choice in a JSON file keyed by device, operator, order and problem size, so later runs of the
same shape skip the search.

Timing runs stage 0 of the LSERK4 scheme with dt = 0 from a step boundary: the residual becomes 0 and the
state is rewritten unchanged, so tuning leaves the solution where it was (the next real stage 0 ignores the
residual).  Every candidate computes the same arithmetic per element, so the choice changes speed only.

Candidates of the mixed stage: its FP32-FMA form with 4, 8 or 11 consumer warps per CTA and a ring of as many
slots as shared memory holds, or 6; and, at orders 1..4, its tensor-core form with 2 or 4 threads per element
(8 or 16 consumer warps).  The two forms round differently (both within the mixed stage's error bound); launch
shapes of one form give the same bits.  The plain stages have one launch shape per order and are not tuned.
"""
from __future__ import annotations

import json
import os
import time
from typing import Callable, Dict, List, Optional

from .burgers import RK4B

MIXED_CANDIDATES: List[Dict] = [{"warps": w, "ring": r, "mma": False} for w in (11, 8, 4) for r in (None, 6)]
TCM_CANDIDATES: List[Dict] = [{"warps": w, "ring": None, "mma": True} for w in (16, 8)]


def candidates_for(problem) -> List[Dict]:
    """The launch shapes the tuner tries for this problem's stage operator."""
    return MIXED_CANDIDATES + (TCM_CANDIDATES if problem.N <= 4 else [])


def default_cache_path() -> str:
    env = os.environ.get("DGK_TUNE_CACHE")
    if env:
        return env
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "dgkernel_b200", "tune.json")


def problem_key(device: str, op: str, order: int, dofs: int, parts: int) -> str:
    """Cache key: device name, operator, order, and the problem size rounded to a power of two (DOFs and
    partitions), so nearby sizes share an entry."""
    bucket = 1 << max(0, int(dofs).bit_length() - 1)
    pb = 1 << max(0, int(parts).bit_length() - 1)
    return f"{device}|{op}|N{order}|dofs~{bucket}|parts~{pb}"


def load_cache(path: str) -> dict:
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(path: str, cache: dict) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + f".{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def search(candidates: List[Dict], measure: Callable[[Dict], float]) -> tuple:
    """Measure every candidate (ms per stage) and return (best candidate, {repr: ms})."""
    times = {}
    best, best_ms = None, float("inf")
    for c in candidates:
        ms = float(measure(c))
        times[json.dumps(c, sort_keys=True)] = ms
        if ms < best_ms:
            best, best_ms = c, ms
    return best, times


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "cuda device"


def autotune(problem, cache_path: Optional[str] = None, stages: int = 8, candidates: Optional[List[Dict]] = None,
             force: bool = False) -> Dict:
    """Pick the fastest launch shape of the problem's stage operator, rebuild the operator with it and return
    it ({"warps": .., "ring": ..}).  A cached choice is used unless `force`."""
    if not problem.mixed:
        return {}
    if problem.stage % 5:
        raise ValueError("tune at a step boundary (stage index a multiple of 5)")
    path = cache_path or default_cache_path()
    cache = load_cache(path)
    key = problem_key(_device_name(), "rhsStageMixed", problem.N, problem.dofs, len(problem.Kpart))
    if not force and key in cache:
        best = cache[key]["best"]
        problem.build_stage(**best)
        return best
    r = problem.runner
    if stages % 2:
        stages += 1  # an even count keeps the ping-pong buffers where they were

    def measure(c):
        # stream-synchronised host clock around `stages` launches: enough to rank shapes of a stage that
        # takes much longer than a launch
        problem.build_stage(**c)
        r.ExecuteKernel("rhsStage", 0.0, RK4B[0], 0.0)  # warm-up (module load, attributes)
        r.ExecuteKernel("rhsStage", 0.0, RK4B[0], 0.0)
        r.Sync()
        t0 = time.perf_counter()
        for _ in range(stages):
            r.ExecuteKernel("rhsStage", 0.0, RK4B[0], 0.0)
        r.Sync()
        return (time.perf_counter() - t0) * 1e3 / stages

    best, times = search(candidates or candidates_for(problem), measure)
    problem.build_stage(**best)
    r.Sync()
    cache[key] = {"best": best, "ms_per_stage": times, "when": time.strftime("%Y-%m-%d %H:%M:%S")}
    save_cache(path, cache)
    return best

