"""The replicas path of bench.py on CPU: two gloo ranks (127.0.0.1) check the cross-rank
barrier, max (device time) and sum (rays), and that the reference arm lets ranks other than 0
exit without work."""

import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    reps = bench.Replicas(dist, "cpu")
    reps.barrier()
    ms = reps.max(10.0 + rank)            # the slowest rank's time
    rays = reps.sum(1000.0 * (rank + 1))  # every rank's rays
    reps.close()
    q.put((rank, ms, rays))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
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
    assert got == [(0, 11.0, 3000.0), (1, 11.0, 3000.0)]


def test_single_process_is_identity():
    sys.path.insert(0, REPO)
    import bench
    reps = bench.Replicas(None)
    assert reps.max(3.5) == 3.5 and reps.sum(7) == 7
    reps.barrier()
    reps.close()


def test_reference_arm_other_ranks_exit(monkeypatch):
    sys.path.insert(0, REPO)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("A", (), {"steps": 1, "warmup": 0, "gpus": 2})()
    assert bench.run_reference(args, bench.WORKLOADS["c2"]) == 0
