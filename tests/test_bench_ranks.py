"""The N > 1 path of bench.py on CPU: two gloo ranks run the replica
aggregation (barrier, max over ranks of the step time, whole-job rate) and
the reference arm's rank rule (only rank 0 reports)."""
from __future__ import annotations

import os
import sys

import pytest
import torch.multiprocessing as mp


def _rank_main(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench._barrier(world)
        # rank r "took" 2 + r ms for 1,000 units: the job is as slow as rank 1
        rate, ms = bench.replica_rate(world, 1000.0, 2.0 + rank)
        args = type("A", (), {"steps": 1, "warmup": 0, "workload": "plain"})()
        ref = bench.run_reference(args) if rank != 0 else "rank0"
        out.put((rank, rate, ms, ref))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_the_driver():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, rate, ms, ref in res:
        assert ms == pytest.approx(3.0)                     # max over ranks
        assert rate == pytest.approx(2000.0 / 3.0e-3)       # all units / slowest time
    assert res[1][3] is None                                # rank 1 of the reference arm prints nothing
