"""Multi-GPU runs of bench.py are independent replicas (the time step has no
inter-GPU exchange on one domain): the process group only synchronises the
timed region and takes the slowest replica's time. Checked here with two
gloo ranks on the CPU: the torchrun environment is read, the max-over-ranks
reduction gives every rank the largest time, the job throughput counts every
replica, and the reference arm does its work on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, dist = bench.dist_setup(world, backend="gloo")
    try:
        dist.barrier()
        t = bench.max_over_ranks(10.0 + 5.0 * r, dist, "cpu")
        out.put((r, w, local, t, bench.replica_mlups(1_000_000, 100, t, w)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1] and all(g[1] == 2 for g in got)
    assert all(g[3] == 15.0 for g in got)  # the slower replica's time
    assert all(g[4] == pytest.approx(2 * 1_000_000 * 100 / 0.015 / 1e6) for g in got)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
