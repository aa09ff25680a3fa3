"""The multi-GPU path of bench.py on the CPU: replicas only (every rank advances the whole
workload on its own GPU, no data-path collective), joined by a barrier and timed by the slowest
rank. Two gloo ranks check the barrier, the maximum over ranks and the job's throughput, and the
reference arm's other ranks exit without work."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.replica_barrier(world, device="cpu")
        ms = bench.replica_max(10.0 + rank, world, device="cpu")  # rank 1 is the slower replica
        out.put((rank, ms, bench.replica_value(1000, 20, ms, world)))
        bench.replica_barrier(world, device="cpu")
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, value in got:
        assert ms == 11.0
        assert abs(value - 2 * 1000 * 20 / 11.0e-3) <= 1e-6 * value


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, env=env, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
