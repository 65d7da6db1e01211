"""The N-GPU bench path on CPU: replicas time their own region and rank 0 reports the
whole-job throughput against the slowest rank (world size 2, gloo)."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 50.0 * rank            # rank 1 is the slow replica
        ms_max = bench.max_over_ranks(ms, world)
        out[rank] = (ms_max, bench.replica_throughput(world, 1000, 10, ms_max))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_world2():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    # every rank sees the slowest replica's time; throughput counts both replicas' work
    assert res[0][0] == res[1][0] == 150.0
    assert abs(res[0][1] - 2 * 1000 * 10 / 0.150) < 1e-6


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_throughput(1, 998582, 10, 219.4) == 998582 * 10 / 0.2194


def test_bench_refuses_a_world_size_other_than_gpus():
    """`--gpus N` under a launcher with another world size would time the wrong number of
    replicas: bench.py refuses before any GPU work."""
    import subprocess
    env = dict(os.environ, WORLD_SIZE="3", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--steps", "1"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 2
    assert "WORLD_SIZE is 3" in r.stderr
