"""The multi-GPU path of bench.py is replicas only: every rank solves its own
system and the job's throughput is the units summed over ranks over the
slowest rank's time.  Checked here on CPU with two gloo ranks."""
import os
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t_ms = [120.0, 150.0][rank]
        units = [30, 28][rank]
        q.put((rank, bench.replica_throughput(t_ms, units, dist, "cpu")))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        t_max, total, value = out[r]
        assert t_max == 150.0 and total == 58
        assert value == pytest.approx(58 / 0.150)


def test_replicas_are_independent_systems():
    sys.path.insert(0, ROOT)
    import bench

    a, b = bench.Workload("monolayer", 0), bench.Workload("monolayer", 1)
    assert a.pos.shape == b.pos.shape
    assert not (a.eps == b.eps).all()   # own frequency set per rank


def test_single_process_throughput():
    sys.path.insert(0, ROOT)
    import bench

    t, n, v = bench.replica_throughput(50.0, 30)
    assert (t, n) == (50.0, 30) and v == pytest.approx(600.0)
