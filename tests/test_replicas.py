"""Multi-GPU form of the benchmark (independent replicas, one process per GPU): the timing of a
step is the slowest rank's and the whole-job rate counts every rank's solves.  Exercised here with
two gloo ranks on the CPU; the reference arm does its work on rank 0 only."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 100.0 * (rank + 1)          # rank 1 is the slow one
        t = bench.max_over_ranks(local_ms, dist, "cpu")
        rate = bench.replica_rate(3, world, t / 1e3)
        q.put((rank, t, rate))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, rate in res:
        assert t == 200.0                       # max over ranks
        assert rate == pytest.approx(2 * 3 / 0.2)


def test_single_process_has_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.replica_rate(4, 1, 2.0) == 2.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        steps, warmup = 1, 0
    bench.reference_main(Args(), 2, 1)         # rank 1 of 2: returns without work or output
    assert capsys.readouterr().out == ""
