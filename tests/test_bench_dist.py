"""World-size-2 plumbing of bench.py on the host (gloo ranks, no GPU): rank setup from the torchrun
environment, the barrier and the max over ranks that bracket every timed region, and the reference arm,
which rank 0 alone runs and prints while the other ranks exit 0 without work."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(script, *args, timeout=300):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2", "--master-addr",
           "127.0.0.1", "--master-port", str(_port()), script, *args]
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env, cwd=ROOT)


def test_rank_setup_barrier_and_max_over_ranks(tmp_path):
    script = tmp_path / "ranks.py"
    script.write_text(
        "import sys\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "import bench\n"
        "world, rank, local = bench.dist_setup(None)\n"
        "bench.barrier(world)\n"
        "m = bench.max_over_ranks(1.5 * (rank + 1), world)\n"
        f"open({str(tmp_path)!r} + f'/rank{{rank}}.txt', 'w').write(f'RANK {{rank}} WORLD {{world}} LOCAL {{local}} MAX {{m}}')\n"
        "bench.barrier(world)\n"
        "import torch.distributed as dist\n"
        "dist.destroy_process_group()\n")
    r = _torchrun(str(script))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [(tmp_path / f"rank{k}.txt").read_text() for k in (0, 1)]
    assert lines == ["RANK 0 WORLD 2 LOCAL 0 MAX 3.0", "RANK 1 WORLD 2 LOCAL 1 MAX 3.0"]


def test_reference_arm_two_ranks_prints_once():
    r = _torchrun("bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--order", "2",
                  "--cubes", "8", "--slabs", "4")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["serial"]["cores"] == 1 and d["cpu_baseline"]["serial"]["value"] > 0
    assert "8^3x6" in d["config"]["workload"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
