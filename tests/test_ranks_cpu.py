"""The multi-process path of bench.py on the CPU (gloo, world size 2).

bench.py runs one process per GPU under torchrun; each rank advances its own
replica (weak scaling, no collective on the data path) and the reported time
is the max over ranks.  Here two CPU processes exercise the same rank helper
(`bench.Ranks`) over gloo, and the reference arm is launched through torchrun
with two ranks: only rank 0 works and prints, the other exits 0.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks("gloo", "cpu")
    r.barrier()
    # device-timed values differ per rank; everyone must see the slowest
    slowest = r.max(10.0 + rank)
    job = r.whole_job_mlups(1000, 10, slowest)
    r.barrier()
    r.close()
    q.put((rank, slowest, job))


def test_max_over_ranks_gloo_world_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, slowest, job in got:
        assert slowest == 11.0
        # 2 ranks x 1000 nodes x 10 steps over 11 ms
        assert job == pytest.approx(2 * 1000 * 10 / 11e-3 / 1e6)


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--lattice", "256", "256"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] == 1
    assert d["config"]["lattice"] == [256, 256] and "reduced" in d["config"]["workload"]
    assert d["cpu_baseline"]["cpu_model"] and d["cpu_baseline"]["pinned_core"] is not None


def test_bench_gpus_two_launches_its_own_ranks():
    """`bench.py --gpus 2` without torchrun starts both rank processes itself."""
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "2",
           "--warmup", "3", "--lattice", "128", "128"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["config"]["timed_steps"] == 2
